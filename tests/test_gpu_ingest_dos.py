"""GPU parity for matrix ingestion (COO -> CSR -> SELL-32 on the device), the
Lanczos DOS and the reference's Matrix-Market pipeline (TESTS/PLanN/MMPLanN.c:
LanTrbounds -> LanDos -> spslicer2 -> ChebLanNr per slice) on its own test
matrix A.mtx.

Tolerances: device COO -> CSR and SpMV bitwise; LanDos curve within 1e-10
relative (the reorthogonalisation differs from the reference's modified
Gram-Schmidt by rounding only), its count within 1e-9 relative; slices equal
to the reference's when the curves cross the thresholds at the same grid
points; eigenvalue counts per slice exact, eigenvalues within 1e-10 x
(spectral width) of the reference's and of the dense eigensolver's.
"""
import gzip
import os
import shutil

import numpy as np
import pytest

import evsl_b200 as E
from oracle import evsl_oracle as O

pytestmark = pytest.mark.gpu

MM_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mm")


@pytest.fixture(scope="module")
def a_mtx(tmp_path_factory):
    p = tmp_path_factory.mktemp("mm") / "A.mtx"
    with gzip.open(os.path.join(MM_DIR, "A.mtx.gz"), "rb") as src, open(p, "wb") as dst:
        shutil.copyfileobj(src, dst)
    return str(p)


@pytest.mark.parametrize("name", ["gen_dup", "int_upper", "skew", "sym"])
@pytest.mark.parametrize("on_device", [False, True])
def test_device_coo_to_csr_matches_reference(gpu_lib, golden, name, on_device):
    coo = golden[f"mm_{name}_coo"]
    vv = golden[f"mm_{name}_vv"]
    n = len(golden[f"mm_{name}_ia"]) - 1
    for base in (0, 1):
        csr = gpu_lib.coo_to_csr_device(n, coo[0] + base, coo[1] + base, vv, base, on_device)
        ia, ja, a = gpu_lib.csr_device_to_host(csr)
        gpu_lib.free_csr_device(csr)
        assert np.array_equal(ia, golden[f"mm_{name}_ia"])
        assert np.array_equal(ja, golden[f"mm_{name}_ja"])
        assert np.array_equal(a, golden[f"mm_{name}_a"])


def test_device_coo_to_csr_large_irregular(gpu_lib):
    """Duplicates, empty rows, a 70,000-entry row and far-off-diagonal
    columns; compared with the stable sort of the oracle."""
    rng = np.random.default_rng(8)
    n, m = 200_000, 1_500_000
    r = rng.integers(0, n, m)
    c = rng.integers(0, n, m)
    r[:70_000] = 12345
    r[70_000:70_100] = r[70_100:70_200]
    c[70_000:70_100] = c[70_100:70_200]
    r[(r > 1000) & (r < 1100)] = 5
    v = rng.standard_normal(m)
    csr = gpu_lib.coo_to_csr_device(n, r, c, v, 0, True)
    got = gpu_lib.csr_device_to_host(csr)
    gpu_lib.free_csr_device(csr)
    ref = O.coo_to_csr(n, r, c, v, 0)
    assert all(np.array_equal(g, x) for g, x in zip(got, ref))


def test_device_coo_to_csr_rejects_bad_index(gpu_lib):
    with pytest.raises(E.EvslError):
        gpu_lib.coo_to_csr_device(10, [0, 3, 10], [0, 1, 2], [1.0, 2.0, 3.0], 0, True)
    with pytest.raises(E.EvslError):
        gpu_lib.coo_to_csr_device(10, [1, 3, 5], [0, 1, 2], [1.0, 2.0, 3.0], 1, False)


def test_set_coo_spmv_bitwise_and_storage(gpu_lib):
    """Matrices registered through device ingestion: every storage format of
    the SELL-32 build (float/double values, int16/int32 column offsets)."""
    rng = np.random.default_rng(3)
    n = 70_000
    for far, float_vals in ((False, True), (True, True), (False, False), (True, False)):
        m = 8 * n
        r = rng.integers(0, n, m)
        c = np.clip(r + rng.integers(-50, 51, m), 0, n - 1)
        if far:
            c[::97] = np.where(r[::97] < n - 33_000, r[::97] + 33_000, r[::97] - 33_000)
        v = rng.integers(-8, 9, m).astype(np.float64) if float_vals else rng.standard_normal(m)
        r = np.concatenate([r, np.arange(n)])
        c = np.concatenate([c, np.arange(n)])
        v = np.concatenate([v, np.full(n, 20.0)])
        gpu_lib.set_coo(n, r, c, v, 0, True)
        vb, ib = gpu_lib.matrix_storage()
        assert vb == (4 if float_vals else 8) and ib == (4 if far else 2)
        ia, ja, a = O.coo_to_csr(n, r, c, v, 0)
        x = rng.standard_normal(n)
        assert np.array_equal(gpu_lib.matvec(x), O.csr_matvec(ia, ja, a, x))


def test_lan_dos_matches_reference(gpu_lib, golden):
    ia, ja, a = O.lap_csr(30, 30, 1)
    gpu_lib.set_csr(ia, ja, a)
    gpu_lib.set_seed(11)
    x, y, ec = gpu_lib.lan_dos(10, 40, 200, [0.5, 2.0, 0.0, 8.0])
    assert np.array_equal(x, golden["ld30_x"])
    assert np.max(np.abs(y - golden["ld30_y"])) <= 1e-10 * np.max(np.abs(golden["ld30_y"]))
    assert abs(ec - golden["ld30_ecnt"][0]) <= 1e-9 * golden["ld30_ecnt"][0]
    assert np.array_equal(E.spslicer2(x, y, 4), golden["ld30_sli"])


def test_mm_pipeline_on_reference_matrix(gpu_lib, golden, a_mtx):
    """TESTS/PLanN/MMPLanN.c on MATRICES/A.mtx: [0.1, 0.3] in 5 slices,
    LanDos with 30 vectors x 80 steps, ChebLanNr tol 1e-6 in each slice."""
    n, ir, jc, vv = E.read_coo_mm(a_mtx, 1, 0)
    gpu_lib.set_coo(n, ir, jc, vv, 0, False)
    vinit = O.library_uniform(2024, 0, n)
    lo, hi = gpu_lib.lan_trbounds(50, 200, 1e-8, vinit, 1)
    ref_lo, ref_hi = golden["mmA_bounds"]
    assert abs(lo - ref_lo) <= 1e-7 * (abs(ref_lo) + abs(ref_hi))
    assert abs(hi - ref_hi) <= 1e-7 * (abs(ref_lo) + abs(ref_hi))
    ex_lo, ex_hi = golden["mmA_extremes"]
    assert lo <= ex_lo + 1e-9 and hi >= ex_hi - 1e-9
    gpu_lib.set_seed(77)
    x, y, ec = gpu_lib.lan_dos(30, 80, 500, [0.1, 0.3, lo, hi])
    assert abs(ec - golden["mmA_ecnt"][0]) <= 1e-9 * golden["mmA_ecnt"][0]
    sli = E.spslicer2(x, y, 5)
    assert np.array_equal(sli, golden["mmA_sli"])
    found = []
    for s in range(5):
        nev = int(1.2 * int(1 + ec / 5))
        mlan = min(max(5 * nev, 300), n)
        xi = [sli[s], sli[s + 1], lo, hi]
        pol = gpu_lib.find_pol(xi, damping=2, thresh_int=0.8, thresh_ext=0.2)
        lam, Y, res = gpu_lib.cheblan_nr(xi, mlan, 1e-6, vinit, pol, want_vectors=False)
        gpu_lib.free_pol(pol)
        assert len(lam) == golden["mmA_counts"][s]
        assert np.all(res < 1e-6)
        found.append(np.sort(lam))
    found = np.concatenate(found)
    width = ex_hi - ex_lo
    assert np.max(np.abs(found - golden["mmA_lam"])) <= 1e-10 * width
    assert np.max(np.abs(found - golden["mmA_exact"])) <= 1e-10 * width
