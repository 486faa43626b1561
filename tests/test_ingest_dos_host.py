"""Host-side parity (no GPU): the library's Matrix-Market reader, COO -> CSR,
simpson, spslicer2 and exDOS against the reference build's outputs on the
committed fixtures, and the oracle's restatements of the same functions.

Tolerances: reader, COO -> CSR, simpson, spslicer2 and exDOS bitwise (same
host arithmetic); the oracle's LanDos restatement within 1e-12 relative of
the reference's DOS curve (dot-product order and the tridiagonal eigensolver
differ).
"""
import gzip
import os
import shutil

import numpy as np
import pytest

import evsl_b200 as E
from oracle import evsl_oracle as O

MM_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mm")
MM_CASES = ["gen_dup", "int_upper", "pattern", "rect", "short", "skew", "sym"]


def mm_path(name):
    return os.path.join(MM_DIR, name + ".mtx")


@pytest.fixture(scope="module")
def a_mtx(tmp_path_factory):
    """The reference's stiffness matrix A.mtx, decompressed."""
    p = tmp_path_factory.mktemp("mm") / "A.mtx"
    with gzip.open(os.path.join(MM_DIR, "A.mtx.gz"), "rb") as src, open(p, "wb") as dst:
        shutil.copyfileobj(src, dst)
    return str(p)


@pytest.mark.parametrize("name", MM_CASES)
def test_mm_reader_matches_reference(golden, name):
    rc_ref = int(golden[f"mm_{name}_rc"][0])
    if rc_ref != 0:
        with pytest.raises(E.EvslError, match=f"returned {rc_ref}"):
            E.read_coo_mm(mm_path(name), 1, 0)
        assert O.read_coo_mm(mm_path(name), 1, 0)[0] == rc_ref
        return
    n, ir, jc, vv = E.read_coo_mm(mm_path(name), 1, 0)
    coo = golden[f"mm_{name}_coo"]
    assert np.array_equal(ir, coo[0]) and np.array_equal(jc, coo[1])
    assert np.array_equal(vv, golden[f"mm_{name}_vv"])
    rc, n2, ir2, jc2, vv2 = O.read_coo_mm(mm_path(name), 1, 0)
    assert rc == 0 and n2 == n and np.array_equal(ir2, ir) and np.array_equal(jc2, jc) and np.array_equal(vv2, vv)
    # one-based output keeps the file's indices
    n1, ir1, jc1, _ = E.read_coo_mm(mm_path(name), 1, 1)
    assert np.array_equal(ir1, ir + 1) and np.array_equal(jc1, jc + 1)


@pytest.mark.parametrize("name", ["gen_dup", "int_upper", "skew", "sym"])
def test_coo_to_csr_host_matches_reference(golden, name):
    coo = golden[f"mm_{name}_coo"]
    vv = golden[f"mm_{name}_vv"]
    n = len(golden[f"mm_{name}_ia"]) - 1
    ref = (golden[f"mm_{name}_ia"], golden[f"mm_{name}_ja"], golden[f"mm_{name}_a"])
    for got in (E.coo_to_csr_host(n, coo[0], coo[1], vv, 0), O.coo_to_csr(n, coo[0], coo[1], vv, 0),
                E.coo_to_csr_host(n, coo[0] + 1, coo[1] + 1, vv, 1)):
        assert all(np.array_equal(g, r) for g, r in zip(got, ref))


def test_coo_to_csr_host_rejects_bad_indices():
    with pytest.raises(E.EvslError):
        E.coo_to_csr_host(4, [0, 4], [0, 1], [1.0, 2.0], 0)


def test_reference_matrix_reads_identically(a_mtx):
    n, ir, jc, vv = E.read_coo_mm(a_mtx, 1, 0)
    rc, n2, ir2, jc2, vv2 = O.read_coo_mm(a_mtx, 1, 0)
    assert rc == 0 and n == n2 == 5795 and len(ir) == 136565
    assert np.array_equal(ir, ir2) and np.array_equal(jc, jc2) and np.array_equal(vv, vv2)
    ia, ja, a = E.coo_to_csr_host(n, ir, jc, vv, 0)
    ia2, ja2, a2 = O.coo_to_csr(n, ir, jc, vv, 0)
    assert np.array_equal(ia, ia2) and np.array_equal(ja, ja2) and np.array_equal(a, a2)


def test_simpson_spslicer2_exdos_bitwise(golden):
    x, y = golden["ld30_x"], golden["ld30_y"]
    assert np.array_equal(E.spslicer2(x, y, 4), golden["ld30_sli"])
    assert np.array_equal(O.spslicer2(x, y, 4), golden["ld30_sli"])
    assert np.array_equal(E.simpson(x, y), O.simpson(x, y))
    vals = O.exeiglap3(30, 30, 1, 0.0, 8.0)
    rc, xe, ye = E.exdos(vals, 300, [0.5, 2.0, 0.0, 8.0])
    assert rc == 0 and np.array_equal(ye, golden["exdos30_y"])
    rc2, xe2, ye2 = O.exdos(vals, 300, [0.5, 2.0, 0.0, 8.0])
    assert rc2 == 0 and np.array_equal(ye2, golden["exdos30_y"])
    # npts odd and even, a single interval
    for npts in (7, 8):
        xx = O.linspace(0.0, 1.0, npts)
        yy = np.cos(xx)
        assert np.array_equal(E.simpson(xx, yy), O.simpson(xx, yy))
        assert np.array_equal(E.spslicer2(xx, yy, 1), O.spslicer2(xx, yy, 1))


def test_lan_dos_restatement(golden):
    ia, ja, a = O.lap_csr(30, 30, 1)
    x, y, ec = O.lan_dos(10, 40, 200, [0.5, 2.0, 0.0, 8.0], ia, ja, a, 11)
    assert np.array_equal(x, golden["ld30_x"])
    assert np.max(np.abs(y - golden["ld30_y"])) <= 1e-12 * np.max(np.abs(golden["ld30_y"]))
    assert abs(ec - golden["ld30_ecnt"][0]) <= 1e-12 * abs(golden["ld30_ecnt"][0])
