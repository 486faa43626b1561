"""SELL-C-sigma storage and the general sparse matrices it is for.

The random sparse SPD generator of the mixed-precision configuration (16
seeded off-diagonal columns per row, symmetrised, diagonally dominant) gives
rows of 18-54 entries; chunks of 32 consecutive rows then carry ~27% padding,
and sorting the rows of each window of 256 rows by length (SELL-C-sigma) cuts
it to ~4%.  The sort only moves rows between slots: every row keeps its CSR
order, vectors keep the caller's order, so every filter and matvec result is
bitwise the reference's CPU arithmetic (SRC/spmat.c:257-298 matvec_csr,
SRC/chebpoly.c:519-598 ChebAv), whatever the window.

Tolerances: bitwise for SpMV, ChebAv and the FP64 multi-column filter;
FP32 filter 1e-4 relative to the FP64 result (degree 60); eigenvalues within
1e-10 x spectral width (FP64) and 1e-8 x width (mixed) of the reference build's
and the dense solver's, counts exact, residuals below tol.
"""
import numpy as np
import pytest

import evsl_b200 as E
from evsl_b200 import workloads as W
from oracle import evsl_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rspd():
    # 20,013 rows: not a multiple of 32 nor of any sort window
    ia, ja, a = W.random_spd_csr(20013, 16, 33)
    return ia, ja, a


def _register(lib, sigma, ia, ja, a):
    lib.set_sell_sigma(sigma)
    try:
        lib.set_csr(ia, ja, a)
    finally:
        lib.set_sell_sigma(-1)
    return lib.matrix_sell_layout()


def test_sigma_layout_choice(gpu_lib, rspd):
    ia, ja, a = rspd
    nnz = int(ia[-1])
    sigma, stored, plain = _register(gpu_lib, -1, ia, ja, a)
    assert sigma == 256
    assert plain > 1.2 * nnz and stored < 1.06 * nnz
    sigma, stored0, plain0 = _register(gpu_lib, 0, ia, ja, a)
    assert sigma == 0 and stored0 == plain0 == plain
    # a Laplacian's chunks are already full: the automatic choice keeps them
    sigma, stored, plain = _register(gpu_lib, -1, *O.lap_csr(17, 13, 11))
    assert sigma == 0 and stored == plain
    with pytest.raises(E.EvslError):
        gpu_lib.set_sell_sigma(48)


@pytest.mark.parametrize("sigma", [-1, 0, 32, 256, 2048])
def test_sigma_spmv_and_filter_bitwise(gpu_lib, rspd, sigma):
    ia, ja, a = rspd
    n = len(ia) - 1
    _register(gpu_lib, sigma, ia, ja, a)
    x = O.seeded_normal(n, 5)
    assert np.array_equal(gpu_lib.matvec(x), O.csr_matvec(ia, ja, a, x))
    lo, hi = W.gershgorin_bounds(ia, ja, a)
    iv = [lo + 0.3 * (hi - lo), lo + 0.33 * (hi - lo), lo, hi]
    pol = gpu_lib.find_pol(iv, deg=60)
    y_ref = O.cheb_av(O.find_pol(iv, deg=60), ia, ja, a, x)
    try:
        assert np.array_equal(gpu_lib.chebav(pol, x), y_ref)
        # two rows per thread and the single-launch cooperative filter
        gpu_lib.lib.evslx_set_filter_rows_per_thread(2)
        assert np.array_equal(gpu_lib.chebav(pol, x), y_ref)
        gpu_lib.lib.evslx_set_filter_rows_per_thread(1)
        gpu_lib.set_filter_persistent(True)
        assert np.array_equal(gpu_lib.chebav(pol, x), y_ref)
        gpu_lib.set_filter_persistent(False)
        # the multi-column filter: FP64 bitwise per column, FP32 close
        X = np.stack([x, O.seeded_normal(n, 6), O.seeded_normal(n, 7)])
        Y64 = gpu_lib.chebav_multi([pol] * 3, X, E.PREC_FP64)
        assert np.array_equal(Y64[0], y_ref)
        for c in (1, 2):
            assert np.array_equal(Y64[c], O.cheb_av(O.find_pol(iv, deg=60), ia, ja, a, X[c]))
        Y32 = gpu_lib.chebav_multi([pol] * 3, X, E.PREC_MIXED)
        assert np.max(np.abs(Y32 - Y64)) <= 1e-4 * np.max(np.abs(Y64))
    finally:
        gpu_lib.lib.evslx_set_filter_rows_per_thread(1)
        gpu_lib.set_filter_persistent(False)
        gpu_lib.free_pol(pol)


def test_sigma_irregular_and_empty_rows(gpu_lib):
    """Rows of 0..70 entries (empty rows included), int16 column offsets
    and float values (compressed storage) and the plain forms, every sort
    window: the matvec and the filter stay bitwise."""
    rng = np.random.default_rng(12)
    n = 3001
    rows = []
    for r in range(n):
        k = 0 if r % 17 == 0 else 1 + (r * 37) % 70
        c = np.unique(np.clip(r + rng.integers(-3000, 3000, k), 0, n - 1)) if k else np.zeros(0, np.int64)
        rows.append((c, rng.integers(-8, 9, len(c)).astype(np.float64)))
    ia = np.zeros(n + 1, dtype=np.int32)
    ia[1:] = np.cumsum([len(c) for c, _ in rows])
    ja = np.concatenate([c for c, _ in rows]).astype(np.int32)
    a = np.concatenate([v for _, v in rows])
    x = O.seeded_normal(n, 8)
    iv = [-50.0, 50.0, -600.0, 600.0]
    y_ref = O.cheb_av(O.find_pol(iv, deg=25), ia, ja, a, x)
    for comp in (True, False):
        gpu_lib.set_matrix_compression(comp)
        try:
            for sigma in (-1, 0, 32, 4096):
                got, stored, plain = _register(gpu_lib, sigma, ia, ja, a)
                assert got == sigma if sigma >= 0 else got in (0, 256)
                assert stored <= plain or got == sigma
                assert gpu_lib.matrix_storage() == ((4, 2) if comp else (8, 4))
                assert np.array_equal(gpu_lib.matvec(x), O.csr_matvec(ia, ja, a, x)), (comp, sigma)
                pol = gpu_lib.find_pol(iv, deg=25)
                assert np.array_equal(gpu_lib.chebav(pol, x), y_ref), (comp, sigma)
                gpu_lib.free_pol(pol)
        finally:
            gpu_lib.set_matrix_compression(True)


@pytest.fixture(scope="module")
def golden_scale():
    import os

    return np.load(os.path.join(os.path.dirname(__file__), "golden", "evsl_ref_golden_scale.npz"))


def test_cheblan_nr_random_spd_matches_reference(gpu_lib, golden_scale):
    """ChebLanNr on a 20,000-row matrix of the random SPD generator (the
    mixed-precision configuration's matrix at reduced size), 50 eigenvalues
    from the 1000th up, against the reference build fed the same start
    vector and the dense solver's eigenvalues: FP64 drop-in path (SELL-C-sigma
    storage) and the mixed-precision engine (FP32 filter, FP64 refinement)."""
    G = golden_scale
    ia, ja, a = W.random_spd_csr(int(G["rspd_n"]), 16, int(G["rspd_seed"]))
    n = len(ia) - 1
    iv = list(G["rspd_intv"])
    width = iv[3] - iv[2]
    exact = G["rspd_exact"]
    sigma, _, _ = _register(gpu_lib, -1, ia, ja, a)
    assert sigma == 256
    pol = gpu_lib.find_pol(iv, damping=2, thresh_int=0.8, thresh_ext=0.2)
    assert pol.deg == int(G["rspd_deg"][0])
    v = O.seeded_normal(n, int(G["rspd_vseed"]))
    lam, Y, res = gpu_lib.cheblan_nr(iv, 3000, 1e-8, v, pol, want_vectors=False)
    lam = np.sort(lam)
    assert len(lam) == len(exact) == len(G["rspd_lam"])
    assert np.max(np.abs(lam - G["rspd_lam"])) <= 1e-10 * width
    assert np.max(np.abs(lam - exact)) <= 1e-10 * width
    assert np.all(res < 1e-8)
    gpu_lib.set_mixed_min_rows(0)
    try:
        (lam2, Y2, res2), = gpu_lib.cheblan_nr_batch([iv], 3000, 1e-8, v, [pol], precision=E.PREC_MIXED,
                                                    want_vectors=False)
    finally:
        gpu_lib.set_mixed_min_rows(131072)
    lam2 = np.sort(lam2)
    assert len(lam2) == len(exact)
    assert np.max(np.abs(lam2 - exact)) <= 1e-8 * width
    assert np.all(res2 < 1e-8)
    gpu_lib.free_pol(pol)


@pytest.mark.parametrize("case", ["rspd", "irregular"])
def test_panel_filter_bitwise(gpu_lib, rspd, case):
    """The column-panel kernels (x staged through shared memory panel by
    panel), built here on small matrices by lowering their row threshold:
    several row blocks and panels, odd n (unaligned Lanczos basis columns),
    empty rows.  FP64: the single-vector kernel (variant 7) and the
    multi-column kernel at one column (variant 6) give the reference's
    filtered vector bit for bit, and ChebLanNr gives the same eigenvalues bit
    for bit as with the SELL kernel; FP32 agrees to 1e-4."""
    if case == "rspd":
        ia, ja, a = rspd
    else:
        rng = np.random.default_rng(21)
        n = 6007
        rows = []
        for r in range(n):
            k = 0 if r % 13 == 0 else 1 + (r * 29) % 45
            c = np.unique(rng.integers(0, n, k)) if k else np.zeros(0, np.int64)
            c = np.unique(np.concatenate([c, [r]])) if k else c
            rows.append((c, np.where(c == r, 60.0, rng.uniform(-1, 1, len(c)))))
        ia = np.zeros(n + 1, dtype=np.int32)
        ia[1:] = np.cumsum([len(c) for c, _ in rows])
        ja = np.concatenate([c for c, _ in rows]).astype(np.int32)
        a = np.concatenate([v for _, v in rows])
    n = len(ia) - 1
    lo, hi = W.gershgorin_bounds(ia, ja, a)
    iv = [lo + 0.3 * (hi - lo), lo + 0.34 * (hi - lo), lo, hi]
    x = O.seeded_normal(n, 9)
    y_ref = O.cheb_av(O.find_pol(iv, deg=40), ia, ja, a, x)
    gpu_lib.set_panel_filter(True, 1000, 1024)  # several panels even on these small matrices
    try:
        for variant in (7, 0):
            gpu_lib.set_filter_kernel(variant)
            _register(gpu_lib, 256, ia, ja, a)
            pol = gpu_lib.find_pol(iv, deg=40)
            y = gpu_lib.chebav(pol, x)
            assert np.array_equal(y, y_ref), (variant, np.max(np.abs(y - y_ref)))
            if variant == 7:
                R, Wd, nbytes = gpu_lib.matrix_panel_layout(False)
                assert R > 0 and 0 < Wd < n and nbytes > 0, (R, Wd)
                lam7 = gpu_lib.cheblan_nr(iv, 1500, 1e-8, x, pol, want_vectors=False)[0]
            else:
                lam0 = gpu_lib.cheblan_nr(iv, 1500, 1e-8, x, pol, want_vectors=False)[0]
            gpu_lib.free_pol(pol)
        assert np.array_equal(lam7, lam0)
        gpu_lib.set_filter_kernel(-1)
        pol = gpu_lib.find_pol(iv, deg=40)
        gpu_lib.set_filter_variant(6)
        Y64 = gpu_lib.chebav_multi([pol], x[None, :], E.PREC_FP64)
        assert np.array_equal(Y64[0], y_ref)
        Y32 = gpu_lib.chebav_multi([pol], x[None, :], E.PREC_MIXED)
        assert gpu_lib.matrix_panel_layout(True)[0] > 0
        assert np.max(np.abs(Y32[0] - y_ref)) <= 1e-4 * np.max(np.abs(y_ref))
        gpu_lib.free_pol(pol)
    finally:
        gpu_lib.set_filter_variant(-1)
        gpu_lib.set_filter_kernel(-1)
        gpu_lib.set_panel_filter(True, 1 << 18, 16384)


@pytest.mark.parametrize("ncols, range_kib", [(2, 128), (3, 128), (8, 128), (16, 128), (4, 0)])
def test_column_split_filter_bitwise(gpu_lib, rspd, ncols, range_kib):
    """Filter variant 7 (the column-split copy: column ranges whose rows of
    the block fit a byte budget, each row's running sum carried from range to
    range) on the random SPD matrix, with the budget lowered to 128 KiB so
    that this 20,013-row matrix is cut into 2 to 32 ranges at every width,
    and with the default budget (one range).  Columns
    with their own polynomials (degrees 24-45, some masked early): FP64 is the
    reference's ChebAv of each column bit for bit (rows summed in CSR order,
    padding skipped); FP32 equals the SELL kernel's FP32 result (same fused
    multiply-adds in the same order) and is within 1e-4 of FP64."""
    ia, ja, a = rspd
    n = len(ia) - 1
    lo, hi = W.gershgorin_bounds(ia, ja, a)
    ivs = [[lo + (0.2 + 0.03 * c) * (hi - lo), lo + (0.25 + 0.03 * c) * (hi - lo), lo, hi] for c in range(ncols)]
    degs = [24 + (7 * c) % 22 for c in range(ncols)]
    X = np.stack([O.seeded_normal(n, 40 + c) for c in range(ncols)])
    refs = [O.cheb_av(O.find_pol(ivs[c], deg=degs[c]), ia, ja, a, X[c]) for c in range(ncols)]
    pols = [gpu_lib.find_pol(ivs[c], deg=degs[c]) for c in range(ncols)]
    gpu_lib.set_split_range_bytes(range_kib << 10)
    try:
        _register(gpu_lib, -1, ia, ja, a)
        gpu_lib.set_filter_variant(7)
        Y64 = gpu_lib.chebav_multi(pols, X, E.PREC_FP64)
        for c in range(ncols):
            assert np.array_equal(Y64[c], refs[c]), (c, np.max(np.abs(Y64[c] - refs[c])))
        Y32 = gpu_lib.chebav_multi(pols, X, E.PREC_MIXED)
        assert np.max(np.abs(Y32 - Y64)) <= 1e-4 * np.max(np.abs(Y64))
        gpu_lib.set_filter_variant(0)
        assert np.array_equal(gpu_lib.chebav_multi(pols, X, E.PREC_MIXED), Y32)
        # tuned on a freshly registered matrix: whichever variant wins, FP64 stays bitwise
        gpu_lib.set_filter_variant(-1)
        _register(gpu_lib, -1, ia, ja, a)
        Y = gpu_lib.chebav_multi(pols, X, E.PREC_FP64)
        assert all(np.array_equal(Y[c], refs[c]) for c in range(ncols))
    finally:
        gpu_lib.set_filter_variant(-1)
        gpu_lib.set_split_range_bytes(0)
        for p in pols:
            gpu_lib.free_pol(p)


def test_column_split_needs_increasing_columns(gpu_lib):
    """A row whose column indices are not increasing has no column-split
    copy: forcing variant 7 fails with an error, the tuned filter serves it
    with the SELL kernels in CSR order (bitwise the reference)."""
    ia, ja, a = W.random_spd_csr(3001, 16, 35)
    ja = ja.copy()
    a = a.copy()
    r = 17
    ja[ia[r]:ia[r + 1]] = ja[ia[r]:ia[r + 1]][::-1].copy()
    a[ia[r]:ia[r + 1]] = a[ia[r]:ia[r + 1]][::-1].copy()
    n = len(ia) - 1
    lo, hi = W.gershgorin_bounds(ia, ja, a)
    iv = [lo + 0.3 * (hi - lo), lo + 0.35 * (hi - lo), lo, hi]
    X = np.stack([O.seeded_normal(n, 50 + c) for c in range(4)])
    pol = gpu_lib.find_pol(iv, deg=20)
    ref = O.cheb_av(O.find_pol(iv, deg=20), ia, ja, a, X[0])
    gpu_lib.set_split_range_bytes(16 << 10)
    try:
        _register(gpu_lib, -1, ia, ja, a)
        gpu_lib.set_filter_variant(7)
        with pytest.raises(E.EvslError):
            gpu_lib.chebav_multi([pol] * 4, X, E.PREC_FP64)
        gpu_lib.set_filter_variant(-1)
        _register(gpu_lib, -1, ia, ja, a)
        Y = gpu_lib.chebav_multi([pol] * 4, X, E.PREC_FP64)
        assert np.array_equal(Y[0], ref)
        assert gpu_lib.tuned_filter_variant(E.PREC_FP64, 4) != 7
    finally:
        gpu_lib.set_filter_variant(-1)
        gpu_lib.set_split_range_bytes(0)
        gpu_lib.free_pol(pol)


@pytest.mark.parametrize("nvec", [12, 13])
def test_kpm_on_column_split_copy(gpu_lib, rspd, nvec):
    """The KPM block step on the column-split copy (8 probes at a time, one
    launch per column range, running sums carried between ranges), forced on
    the 20,013-row random SPD matrix with 128 KiB ranges: moments within 1e-12
    (normwise, and per moment relative where |mu_k| >= 1e-3 max |mu|) of the
    reference's direct per-degree recurrence restated in the oracle and of
    the default kernel; even (16-byte loads) and odd probe counts; each
    probe's dot products bitwise the same whichever probes share its block,
    so probe shards reproduce the full block."""
    import ctypes as C

    ia, ja, a = rspd
    n = len(ia) - 1
    lo, hi = W.gershgorin_bounds(ia, ja, a)
    iv = [lo + 0.3 * (hi - lo), lo + 0.36 * (hi - lo), lo, hi]
    M = 60
    probes = O.seeded_rademacher(nvec, n, 71)
    mu_or, ec_or = O.kpmdos(M, 1, probes, iv, ia, ja, a)
    _register(gpu_lib, -1, ia, ja, a)
    mu_def, ec_def = gpu_lib.kpmdos_probes(M, 1, probes, iv)
    gpu_lib.set_split_range_bytes(128 << 10)
    gpu_lib.lib.evslcu_set_kpm_split.argtypes = [C.c_int]
    try:
        _register(gpu_lib, -1, ia, ja, a)
        gpu_lib.lib.evslcu_set_kpm_split(1)
        mu, ec = gpu_lib.kpmdos_probes(M, 1, probes, iv)
        for ref in (mu_or, mu_def):
            assert np.max(np.abs(mu - ref)) <= 1e-12 * np.max(np.abs(ref))
            big = np.abs(ref) >= 1e-3 * np.max(np.abs(ref))
            assert np.all(np.abs(mu - ref)[big] <= 1e-12 * np.abs(ref)[big])
        assert abs(ec - ec_or) <= 1e-10 * abs(ec_or)
        full = E.DeviceBuffer.from_host(gpu_lib.lib, probes)
        dots = gpu_lib.kpm_dots(M, iv, full, nvec)
        for a0, b0 in ((0, 5), (5, nvec)):
            part = E.DeviceBuffer.from_host(gpu_lib.lib, np.ascontiguousarray(probes[a0:b0]))
            assert np.array_equal(gpu_lib.kpm_dots(M, iv, part, b0 - a0), dots[:, a0:b0])
    finally:
        gpu_lib.lib.evslcu_set_kpm_split(-1)
        gpu_lib.set_split_range_bytes(0)
