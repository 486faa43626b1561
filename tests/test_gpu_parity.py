"""GPU parity tests: the CUDA sm_100a library through its C ABI against the
oracle (numpy restatement + golden fixtures from the reference build).

Tolerances (written per test):
  * SpMV and ChebAv (the FP64 filter): bitwise equal to the reference CPU
    arithmetic;
  * KPM moments: normwise ||mu - mu_ref||_inf <= 1e-12 ||mu_ref||_inf (only
    the summation order of the dot products differs); counts to 1e-10;
  * eigenvalues: within 1e-10 x (spectral width) of the reference's, counts
    exact against the analytic Laplacian spectrum, residuals < tol.
"""
import numpy as np
import pytest

from oracle import evsl_oracle as O

pytestmark = pytest.mark.gpu


def _lap(lib, nx, ny, nz):
    ia, ja, a = O.lap_csr(nx, ny, nz)
    lib.set_csr(ia, ja, a)
    return ia, ja, a


@pytest.mark.parametrize("patterns", [True, False])
@pytest.mark.parametrize("kernel", [0, 1])
def test_spmv_bitwise(gpu_lib, kernel, patterns):
    try:
        for dims in ((37, 23, 1), (17, 13, 11)):
            ia, ja, a = _lap(gpu_lib, *dims)
            gpu_lib.set_spmv_kernel(kernel)
            gpu_lib.set_row_patterns(patterns)
            x = np.random.default_rng(5).standard_normal(len(ia) - 1)
            assert np.array_equal(gpu_lib.matvec(x), O.csr_matvec(ia, ja, a, x))
    finally:
        gpu_lib.set_spmv_kernel(0)
        gpu_lib.set_row_patterns(True)


def _csr_from_rows(rows):
    """CSR arrays from a list of (columns, values) per row."""
    ia = np.zeros(len(rows) + 1, dtype=np.int32)
    ia[1:] = np.cumsum([len(c) for c, _ in rows])
    ja = np.concatenate([np.asarray(c, dtype=np.int32) for c, _ in rows] + [np.zeros(0, np.int32)])
    a = np.concatenate([np.asarray(v, dtype=np.float64) for _, v in rows] + [np.zeros(0)])
    return ia, ja, a


@pytest.mark.parametrize("table", ["constant", "global"])
def test_row_pattern_dictionary(gpu_lib, table):
    """The row-pattern dictionary: exact pattern counts on grids, its limit of
    1024 distinct rows, and bitwise SpMV / ChebAv with and without it on rows
    that are empty, hold signed zeros or differ only in one value's last bit,
    with the pattern table read from constant or from global memory."""
    gpu_lib.lib.evslcu_set_pattern_const(1 if table == "constant" else 0)
    try:
        _lap(gpu_lib, 37, 23, 1)
        assert gpu_lib.row_pattern_count() == 9  # corners, edges, interior of a 2-D grid
        _lap(gpu_lib, 17, 13, 11)
        assert gpu_lib.row_pattern_count() == 27
        # a diagonal with 1024 distinct values is kept, with 1025 it is not
        for m, expect in ((1024, 1024), (1025, 0)):
            n = 5000
            d = 1.0 + (np.arange(n) % m)
            gpu_lib.set_csr(np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), d)
            assert gpu_lib.row_pattern_count() == expect, m
            if expect:
                x = np.random.default_rng(2).standard_normal(n)
                assert np.array_equal(gpu_lib.matvec(x), d * x)
        # a 3-D Laplacian with empty rows and explicit +0/-0 entries (values
        # all exactly floats: packed table), and the same with one value
        # changed in its last bit (not a float: unpacked table)
        for tweak in (False, True):
            ia, ja, a = O.lap_csr(12, 11, 10)
            n = len(ia) - 1
            rows = [(list(ja[ia[r]:ia[r + 1]]), list(a[ia[r]:ia[r + 1]])) for r in range(n)]
            for r in range(0, n, 97):
                rows[r] = ([], [])
            for r in range(5, n, 89):
                c, v = rows[r]
                if c:
                    rows[r] = (c, [(-0.0 if k == 0 else x) for k, x in enumerate(v)])
            for r in range(7, n, 83):
                c, v = rows[r]
                if c and tweak:
                    rows[r] = (c, [np.nextafter(v[0], 10.0)] + v[1:])
            ia, ja, a = _csr_from_rows(rows)
            rng = np.random.default_rng(17)
            x = rng.standard_normal(n)
            x[::13] = -0.0
            iv = [0.6, 0.9, 0.0, 12.0]
            y_ref = O.cheb_av(O.find_pol(iv, max_deg=200), ia, ja, a, x)
            for on in (True, False):
                gpu_lib.set_row_patterns(True)  # build the dictionary at registration
                gpu_lib.set_csr(ia, ja, a)
                gpu_lib.set_row_patterns(on)
                if on:
                    assert 0 < gpu_lib.row_pattern_count() <= 1024
                assert np.array_equal(gpu_lib.matvec(x), O.csr_matvec(ia, ja, a, x))
                pol = gpu_lib.find_pol(iv, max_deg=200)
                y = gpu_lib.chebav(pol, x)
                gpu_lib.free_pol(pol)
                assert np.array_equal(y, y_ref), (tweak, on, np.max(np.abs(y - y_ref)))
    finally:
        gpu_lib.set_row_patterns(True)
        gpu_lib.lib.evslcu_set_pattern_const(1)


def test_spmv_irregular_rows(gpu_lib):
    # rows of very different lengths (1 .. 70 entries), unsorted input order irrelevant
    rng = np.random.default_rng(11)
    n = 1000
    rows, cols = [], []
    for r in range(n):
        k = 1 + (r * 37) % 70
        c = np.unique(np.concatenate([[r], rng.integers(0, n, k)]))
        rows += [r] * len(c)
        cols += list(c)
    rows, cols = np.array(rows), np.array(cols)
    vals = rng.standard_normal(len(rows))
    ia = np.zeros(n + 1, dtype=np.int32)
    np.add.at(ia, rows + 1, 1)
    ia = np.cumsum(ia).astype(np.int32)
    gpu_lib.set_csr(ia, cols.astype(np.int32), vals)
    x = rng.standard_normal(n)
    for kernel in (0, 1):
        gpu_lib.set_spmv_kernel(kernel)
        assert np.array_equal(gpu_lib.matvec(x), O.csr_matvec(ia, cols, vals, x))
    gpu_lib.set_spmv_kernel(0)


def test_chebav_matches_reference_golden(gpu_lib, golden):
    _lap(gpu_lib, 20, 20, 1)
    pol = gpu_lib.find_pol([0.6, 1.2, 0.0, 8.0])
    y = gpu_lib.chebav(pol, golden["chebav_v"])
    assert np.array_equal(y, golden["chebav_y"])
    gpu_lib.free_pol(pol)


@pytest.mark.parametrize("kernel", [0, 1])
def test_chebav_bitwise_config_sizes(gpu_lib, kernel):
    # config-1 matrix and filter; and a 3-D case with a degree ~100 filter
    for dims, iv in (((100, 100, 1), [0.6, 0.9, 0.0, 8.0]), ((24, 24, 24), [0.6, 0.69331, 0.0, 12.0])):
        ia, ja, a = _lap(gpu_lib, *dims)
        gpu_lib.set_spmv_kernel(kernel)
        pol = gpu_lib.find_pol(iv, max_deg=3000)
        v = O.seeded_normal(len(ia) - 1, 42)
        y = gpu_lib.chebav(pol, v)
        y_ref = O.cheb_av(O.find_pol(iv, max_deg=3000), ia, ja, a, v)
        assert np.array_equal(y, y_ref), (dims, np.max(np.abs(y - y_ref)))
        gpu_lib.free_pol(pol)
    gpu_lib.set_spmv_kernel(0)


def test_kpmdos_probes_match_reference(gpu_lib, golden):
    _lap(gpu_lib, 20, 20, 1)
    probes = O.seeded_rademacher(6, 400, 7)
    mu, ec = gpu_lib.kpmdos_probes(40, 1, probes, [0.6, 1.2, 0.0, 8.0])
    ref = golden["kpm20_mu"]
    assert np.max(np.abs(mu - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert abs(ec - golden["kpm20_ecnt"][0]) <= 1e-10 * abs(golden["kpm20_ecnt"][0])
    _lap(gpu_lib, 8, 8, 8)
    probes = O.seeded_rademacher(5, 512, 9)
    mu, ec = gpu_lib.kpmdos_probes(60, 1, probes, [0.6, 2.0, 0.0, 12.0])
    ref = golden["kpm8_mu"]
    assert np.max(np.abs(mu - ref)) <= 1e-12 * np.max(np.abs(ref))
    rc, sli = gpu_lib.spslicer(mu, [0.6, 2.0, 0.0, 12.0], 5, int(10 * ec))
    assert rc == 0 and np.max(np.abs(sli - golden["sli8"])) <= 1e-12


def test_kpmdos_many_probes_and_device_rng(gpu_lib):
    # 70 probes (two probe groups) drawn by the library's generator, against
    # the restatement fed the same vectors
    ia, ja, a = _lap(gpu_lib, 15, 11, 3)
    n = len(ia) - 1
    gpu_lib.set_seed(2024)
    mu, ec = gpu_lib.kpmdos(30, 1, 70, [1.0, 3.0, 0.0, 12.0])
    probes = np.stack([O.library_uniform(2024, d, n) for d in range(70)])
    mu_ref, ec_ref = O.kpmdos(30, 1, probes, [1.0, 3.0, 0.0, 12.0], ia, ja, a)
    assert np.max(np.abs(mu - mu_ref)) <= 1e-12 * np.max(np.abs(mu_ref))
    assert abs(ec - ec_ref) <= 1e-10 * abs(ec_ref)


def test_kpm_shards_are_bitwise_the_full_block(gpu_lib):
    """Per-probe dot products do not depend on the other probes of the block,
    so sharding probes over GPUs and accumulating reproduces kpmdos exactly."""
    import evsl_b200

    ia, ja, a = _lap(gpu_lib, 14, 12, 5)
    n = len(ia) - 1
    iv = [0.7, 2.9, 0.0, 12.0]
    gpu_lib.set_seed(99)
    mu_ref, ec_ref = gpu_lib.kpmdos(40, 1, 20, iv)
    full = gpu_lib.draw_probes(n, 0, 20)
    assert np.array_equal(full.to_host(shape=(20, n))[3], O.library_uniform(99, 3, n))
    dots = gpu_lib.kpm_dots(40, iv, full, 20)
    for a0, b0 in ((0, 7), (7, 13), (13, 20)):
        part = gpu_lib.draw_probes(n, a0, b0 - a0)
        assert np.array_equal(gpu_lib.kpm_dots(40, iv, part, b0 - a0), dots[:, a0:b0])
    mu, ec = evsl_b200.kpm_accumulate(40, 1, n, iv, dots)
    assert np.array_equal(mu, mu_ref) and ec == ec_ref


def test_cheblan_nr_small_matches_reference(gpu_lib, golden):
    _lap(gpu_lib, 20, 20, 1)
    pol = gpu_lib.find_pol([0.6, 1.2, 0.0, 8.0])
    lam, Y, res = gpu_lib.cheblan_nr([0.6, 1.2, 0.0, 8.0], 400, 1e-8, golden["chebav_v"], pol)
    ref = golden["nr20_lam"]
    assert len(lam) == len(ref) == len(O.exeiglap3(20, 20, 1, 0.6, 1.2))
    assert np.max(np.abs(np.sort(lam) - ref)) <= 1e-10 * 8.0
    assert np.all(res < 1e-8)
    # eigenvectors: unit norm, mutually orthogonal, A y = lam y
    ia, ja, a = O.lap_csr(20, 20, 1)
    G = Y @ Y.T
    assert np.max(np.abs(G - np.eye(len(lam)))) < 1e-8
    for i in range(len(lam)):
        r = O.csr_matvec(ia, ja, a, Y[i]) - lam[i] * Y[i]
        assert np.linalg.norm(r) < 1e-8
    gpu_lib.free_pol(pol)


def test_cheblan_nr_config1(gpu_lib, golden):
    """Config 1: 2-D 100x100 Laplacian, [0.6, 0.9], thresholds 0.8/0.2,
    tol 1e-8, maxit 2000, seeded normal start vector: 260 eigenpairs."""
    _lap(gpu_lib, 100, 100, 1)
    iv = [0.6, 0.9, 0.0, 8.0]
    pol = gpu_lib.find_pol(iv, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000)
    v = O.seeded_normal(10000, int(golden["cfg1_vinit_seed"][0]))
    lam, Y, res = gpu_lib.cheblan_nr(iv, 2000, 1e-8, v, pol, want_vectors=True)
    exact = O.exeiglap3(100, 100, 1, 0.6, 0.9)
    assert len(lam) == 260 == len(exact)
    lam = np.sort(lam)
    assert np.max(np.abs(lam - golden["cfg1_lam"])) <= 1e-10 * 8.0
    assert np.max(np.abs(lam - exact)) <= 1e-10 * 8.0
    assert np.all(res < 1e-8)
    G = Y @ Y.T
    assert np.max(np.abs(G - np.eye(260))) < 1e-6
    gpu_lib.free_pol(pol)


@pytest.mark.parametrize("grid, iv, maxit", [
    ((100, 100, 1), [0.6, 0.9, 0.0, 8.0], 2000),         # config 1
    ((40, 40, 40), [0.6, 0.8, 0.0, 12.0], 3000),         # tests overlap steps of a larger basis
    ((12, 12, 1), [0.2, 7.8, 0.0, 8.0], 140),            # nearly the whole spectrum, basis near n
    ((40, 40, 1), [0.6, 1.2, 0.0, 8.0], 95),             # maxit reached with a test in flight
])
def test_cheblan_nr_side_stream_tests_bitwise(gpu_lib, grid, iv, maxit):
    """ChebLanNr with its convergence tests on a side stream (the default)
    gives bit for bit what waiting for every test gives: eigenvalues,
    residuals, eigenvectors and the Lanczos dimension."""
    _lap(gpu_lib, *grid)
    n = grid[0] * grid[1] * grid[2]
    pol = gpu_lib.find_pol(iv, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000)
    v = O.seeded_normal(n, 77)
    out = {}
    try:
        for on in (False, True):
            gpu_lib.set_async_tests(on)
            gpu_lib.set_seed(2024)  # lucky breakdowns draw restart vectors from the device RNG
            lam, Y, res = gpu_lib.cheblan_nr(iv, maxit, 1e-8, v, pol, want_vectors=True)
            out[on] = (lam, Y, res, gpu_lib.last_solve_info())
    finally:
        gpu_lib.set_async_tests(True)
        gpu_lib.free_pol(pol)
    a, b = out[False], out[True]
    assert a[3] == b[3]
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


def test_cheblan_tr_small_matches_reference(gpu_lib, golden):
    _lap(gpu_lib, 20, 20, 1)
    pol = gpu_lib.find_pol([0.6, 1.2, 0.0, 8.0])
    lam, Y, res = gpu_lib.cheblan_tr(100, 30, [0.6, 1.2, 0.0, 8.0], 300, 1e-8, golden["chebav_v"], pol)
    ref = golden["tr20_lam"]
    assert len(lam) == len(ref) == len(O.exeiglap3(20, 20, 1, 0.6, 1.2))
    assert np.max(np.abs(np.sort(lam) - ref)) <= 1e-10 * 8.0
    assert np.all(res < 1e-8)
    gpu_lib.free_pol(pol)


def test_cheblan_tr_config1_sized(gpu_lib):
    _lap(gpu_lib, 100, 100, 1)
    iv = [0.6, 0.9, 0.0, 8.0]
    pol = gpu_lib.find_pol(iv, max_deg=3000)
    v = O.seeded_normal(10000, 1234)
    lam, Y, res = gpu_lib.cheblan_tr(1100, 270, iv, 3300, 1e-8, v, pol, want_vectors=False)
    exact = O.exeiglap3(100, 100, 1, 0.6, 0.9)
    assert len(lam) == len(exact)
    assert np.max(np.abs(np.sort(lam) - exact)) <= 1e-10 * 8.0
    assert np.all(res < 1e-8)
    gpu_lib.free_pol(pol)


def test_interval_edge_cases(gpu_lib):
    _lap(gpu_lib, 20, 20, 1)
    pol = gpu_lib.find_pol([0.6, 1.2, 0.0, 8.0])
    v = O.seeded_normal(400, 1)
    # interval outside the spectrum bounds: no eigenpairs, return code 0
    lam, Y, res = gpu_lib.cheblan_nr([9.0, 10.0, 0.0, 8.0], 100, 1e-8, v, pol)
    assert len(lam) == 0
    lam, Y, res = gpu_lib.cheblan_tr(60, 10, [9.0, 10.0, 0.0, 8.0], 100, 1e-8, v, pol)
    assert len(lam) == 0
    # an interval with no eigenvalues inside the spectrum: nothing accepted
    gap = [0.30, 0.3005, 0.0, 8.0]
    assert len(O.exeiglap3(20, 20, 1, gap[0], gap[1])) == 0
    p2 = gpu_lib.find_pol(gap, max_deg=3000)
    lam, Y, res = gpu_lib.cheblan_nr(gap, 200, 1e-8, v, p2)
    assert len(lam) == 0
    gpu_lib.free_pol(p2)
    # end intervals (left and right filters)
    for iv in ([0.0, 0.3, 0.0, 8.0], [7.5, 8.0, 0.0, 8.0]):
        p3 = gpu_lib.find_pol(iv)
        lam, Y, res = gpu_lib.cheblan_nr(iv, 400, 1e-8, v, p3)
        assert len(lam) == len(O.exeiglap3(20, 20, 1, iv[0], iv[1]))
        gpu_lib.free_pol(p3)
    gpu_lib.free_pol(pol)


def test_tiny_problem(gpu_lib):
    # n = 6: Lanczos runs out of dimensions (maxit clipped to n)
    ia, ja, a = _lap(gpu_lib, 3, 2, 1)
    iv = [1.0, 5.0, 0.0, 8.0]
    pol = gpu_lib.find_pol(iv)
    lam, Y, res = gpu_lib.cheblan_nr(iv, 100, 1e-8, O.seeded_normal(6, 2), pol)
    ex = O.exeiglap3(3, 2, 1, iv[0], iv[1])
    assert len(lam) == len(ex)
    assert np.max(np.abs(np.sort(lam) - ex)) < 1e-10
    gpu_lib.free_pol(pol)


@pytest.mark.parametrize("compress", [True, False])
@pytest.mark.parametrize("mode", ["per-degree", "persistent", "wave", "pattern", "pattern-persistent",
                                  "loop-rows"])
def test_filter_variants_bitwise(gpu_lib, compress, mode):
    """Every storage variant (float/double values, int16/int32 columns, the
    row-pattern dictionary) and every execution mode (one launch per degree
    with unrolled or looped row products / one cooperative launch / one
    pipelined launch) give the reference's filtered vector bit for bit."""
    patterns = mode.startswith("pattern")
    gpu_lib.set_matrix_compression(compress)
    gpu_lib.set_filter_persistent(mode.endswith("persistent"))
    gpu_lib.set_filter_wave(mode == "wave")
    gpu_lib.set_row_patterns(patterns)
    gpu_lib.lib.evslcu_set_row_unroll(0 if mode == "loop-rows" else 1)
    try:
        cases = []
        ia, ja, a = O.lap_csr(24, 24, 24)
        cases.append((ia, ja, a, [0.6, 0.69331, 0.0, 12.0]))
        # non-float values and wide bandwidth (forces double values, int32 columns)
        rng = np.random.default_rng(3)
        n = 40000
        rows = np.repeat(np.arange(n), 5)
        cols = np.concatenate([[r, (r + 1) % n, (r * 7919) % n, (r + 35000) % n, (r * 31) % n] for r in range(n)])
        vals = rng.uniform(-1, 1, len(rows)) * 0.1
        key = rows.astype(np.int64) * n + cols
        _, first = np.unique(key, return_index=True)
        rows, cols, vals = rows[first], cols[first], vals[first]
        # symmetric, diagonally dominant
        R = np.concatenate([rows, cols]); Cc = np.concatenate([cols, rows]); V = np.concatenate([vals, vals])
        key = R.astype(np.int64) * n + Cc
        order = np.argsort(key, kind="stable")
        R, Cc, V = R[order], Cc[order], V[order]
        uk, start = np.unique(R.astype(np.int64) * n + Cc, return_index=True)
        V = np.add.reduceat(V, start)
        R, Cc = (uk // n).astype(np.int64), (uk % n).astype(np.int32)
        diag = R == Cc
        V[diag] += 3.0
        ia2 = np.zeros(n + 1, dtype=np.int64)
        np.add.at(ia2, R + 1, 1)
        ia2 = np.cumsum(ia2).astype(np.int32)
        cases.append((ia2, Cc, V, [0.5, 1.0, -1.0, 8.0]))
        for ia, ja, a, iv in cases:
            gpu_lib.set_csr(ia, ja, a)
            vb, ib = gpu_lib.matrix_storage()
            if not compress:
                assert (vb, ib) == (8, 4)
            # the grid has 27 row patterns; the random matrix has no dictionary
            assert gpu_lib.row_pattern_count() == ((27 if ia is cases[0][0] else 0) if patterns else 0)
            pol = gpu_lib.find_pol(iv, max_deg=300)
            v = O.seeded_normal(len(ia) - 1, 9)
            y = gpu_lib.chebav(pol, v)
            y_ref = O.cheb_av(O.find_pol(iv, max_deg=300), ia, ja, a, v)
            assert np.array_equal(y, y_ref), (vb, ib, np.max(np.abs(y - y_ref)))
            gpu_lib.free_pol(pol)
    finally:
        gpu_lib.set_matrix_compression(True)
        gpu_lib.set_filter_persistent(False)
        gpu_lib.set_filter_wave(False)
        gpu_lib.set_row_patterns(True)
        gpu_lib.lib.evslcu_set_row_unroll(1)


@pytest.mark.parametrize("variant", range(7))
def test_filter_kernel_variants_bitwise(gpu_lib, variant):
    """Each single-vector filter kernel, forced, gives the reference's filtered
    vector bit for bit on a grid operator (which has a row-pattern
    dictionary); forcing a pattern kernel on a matrix without one fails with a
    clear error instead of running something else."""
    gpu_lib.set_filter_kernel(variant)
    try:
        iv = [0.6, 0.8, 0.0, 12.0]
        # values all exactly floats (packed pattern table), then a diagonal
        # shifted by 1e-9 every 7th row (double table, 2 patterns more per form)
        for shift in (False, True):
            ia, ja, a = O.lap_csr(23, 21, 19)
            if shift:
                a = a.copy()
                n = len(ia) - 1
                for r in range(0, n, 7):
                    for j in range(ia[r], ia[r + 1]):
                        if ja[j] == r:
                            a[j] += 1e-9
            gpu_lib.set_csr(ia, ja, a)
            assert 0 < gpu_lib.row_pattern_count() <= 1024
            v = O.seeded_normal(len(ia) - 1, 4)
            pol = gpu_lib.find_pol(iv, max_deg=150)
            y = gpu_lib.chebav(pol, v)
            gpu_lib.free_pol(pol)
            assert np.array_equal(y, O.cheb_av(O.find_pol(iv, max_deg=150), ia, ja, a, v)), shift
        # a diagonal with distinct values: no dictionary
        n = 3000
        d = 1.0 + np.arange(n) / n
        gpu_lib.set_csr(np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), d)
        assert gpu_lib.row_pattern_count() == 0
        pol = gpu_lib.find_pol([1.2, 1.5, 1.0, 2.0], max_deg=60)
        x = O.seeded_normal(n, 5)
        if variant >= 2:
            with pytest.raises(Exception, match="not available"):
                gpu_lib.chebav(pol, x)
        else:
            di = np.arange(n + 1, dtype=np.int32)
            y_ref = O.cheb_av(O.find_pol([1.2, 1.5, 1.0, 2.0], max_deg=60), di, di[:-1], d, x)
            assert np.array_equal(gpu_lib.chebav(pol, x), y_ref)
        gpu_lib.free_pol(pol)
    finally:
        gpu_lib.set_filter_kernel(-1)


def test_filter_kernel_is_chosen_by_timing(gpu_lib):
    """With no variant forced, the first filter call times every variant the
    matrix allows and records its choice."""
    _lap(gpu_lib, 30, 30, 30)
    assert gpu_lib.filter_kernel()[0] == -1
    pol = gpu_lib.find_pol([0.6, 0.8, 0.0, 12.0], max_deg=50)
    gpu_lib.chebav(pol, O.seeded_normal(27000, 1))
    gpu_lib.free_pol(pol)
    v, us = gpu_lib.filter_kernel()
    assert len(us) == 7 and v in range(7)
    assert us[gpu_lib.FILTER_KERNELS[v]] == min(us.values())


def test_laplacian_storage_is_compressed(gpu_lib):
    _lap(gpu_lib, 30, 30, 30)
    assert gpu_lib.matrix_storage() == (4, 2)


def test_tridiagonal_eigenvalues_on_gpu(gpu_lib):
    """The convergence tests' tridiagonal eigenvalues (GPU multisection on
    Sturm counts) agree with LAPACK's to 1e-13 of the matrix norm, on sizes
    1..2000, split blocks (exactly repeated eigenvalues), the Wilkinson W21+
    matrix (pairs closer than 1e-13) and tiny off-diagonals."""
    import ctypes as C

    f = gpu_lib.lib.evslcu_trid_eigvals
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(8)
    cases = []
    for k in (1, 2, 3, 64, 65, 500, 2000):
        cases.append((rng.standard_normal(k), rng.standard_normal(max(k - 1, 0))))
    d = np.tile([2.0, -1.0, 0.5], 40)
    e = np.ones(119)
    e[2::3] = 0.0  # 40 identical 3x3 blocks
    cases.append((d, e))
    m = 10
    cases.append((np.abs(np.arange(-m, m + 1)).astype(float), np.ones(2 * m)))  # W21+
    cases.append((np.linspace(0, 1, 300), np.full(299, 1e-170)))
    for d, e in cases:
        d = np.ascontiguousarray(d, dtype=np.float64)
        e = np.ascontiguousarray(e, dtype=np.float64)
        k = len(d)
        w = np.zeros(k)
        assert f(k, d.ctypes.data, e.ctypes.data if k > 1 else None, w.ctypes.data) == 0
        T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
        ref = np.linalg.eigvalsh(T)
        scale = max(np.abs(ref).max(), 1e-300)
        assert np.all(np.diff(w) >= 0)
        assert np.max(np.abs(w - ref)) <= 1e-13 * scale, (k, np.max(np.abs(w - ref)) / scale)


def test_tridiagonal_eigenvalues_above_a_bar(gpu_lib):
    """The trace test's restricted form (only the eigenvalues that may reach
    the bar are computed): every eigenvalue >= xmin is bit for bit the full
    computation's, the entries of the skipped ones lie below xmin, the
    array stays ascending; bars below, inside and above the spectrum, on a
    Lanczos-like spectrum (a cluster of filtered values near 1 over a wide
    bulk) and on repeated eigenvalues."""
    import ctypes as C

    full = gpu_lib.lib.evslcu_trid_eigvals
    full.restype = C.c_int
    full.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    above = gpu_lib.lib.evslcu_trid_eigvals_above
    above.restype = C.c_int
    above.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
    rng = np.random.default_rng(21)
    cases = []
    for k in (64, 300, 3000):
        cases.append((rng.standard_normal(k), rng.standard_normal(k - 1)))
    # tridiagonal with a prescribed spectrum: Lanczos (full reorthogonalisation)
    # on diag(lam), lam = 20% in [0.8, 1], the rest in [-0.1, 0.3]
    n, k = 1500, 400
    lam = np.concatenate([rng.uniform(0.8, 1.0, n // 5), rng.uniform(-0.1, 0.3, n - n // 5)])
    Q = np.zeros((k, n))
    q = rng.standard_normal(n)
    Q[0] = q / np.linalg.norm(q)
    al, be = np.zeros(k), np.zeros(k - 1)
    for j in range(k):
        z = lam * Q[j]
        for _ in range(2):
            z -= Q[: j + 1].T @ (Q[: j + 1] @ z)
        al[j] = Q[j] @ (lam * Q[j])
        if j + 1 < k:
            be[j] = np.linalg.norm(z)
            Q[j + 1] = z / be[j]
    cases.append((al, be))
    d = np.tile([2.0, -1.0, 0.5], 40)
    e = np.ones(119)
    e[2::3] = 0.0
    cases.append((d, e))
    for d, e in cases:
        d = np.ascontiguousarray(d, dtype=np.float64)
        e = np.ascontiguousarray(e, dtype=np.float64)
        k = len(d)
        ref = np.zeros(k)
        assert full(k, d.ctypes.data, e.ctypes.data, ref.ctypes.data) == 0
        for xmin in (ref[0] - 1.0, ref[k // 2], ref[(4 * k) // 5] - 1e-3, 0.8, ref[-1], ref[-1] + 1.0):
            w = np.zeros(k)
            assert above(k, d.ctypes.data, e.ctypes.data, float(xmin), w.ctypes.data) == 0
            keep = ref >= xmin
            assert np.array_equal(w[keep], ref[keep]), (k, xmin)
            assert np.all(w[~keep] < xmin)
            assert np.all(np.diff(w) >= 0)


def test_long_rows_on_the_dictionary(gpu_lib):
    """A banded matrix with 261 entries per interior row keeps a row-pattern
    dictionary (261 row forms, 51,091 table entries) but has rows too long
    for the per-row descriptors and the unrolled forms (16 entries at most),
    and a table too large for the constant-memory pool: the looped SELL-32
    and global-table kernels give the reference's vector bit for bit, and
    every other variant reports that it is not available."""
    n, hb = 2000, 130
    rows = []
    for r in range(n):
        cols = list(range(max(0, r - hb), min(n, r + hb + 1)))
        rows.append((cols, [4.0 * hb if c == r else -1.0 + 0.5 * ((c - r) % 3) for c in cols]))
    ia, ja, a = _csr_from_rows(rows)
    lo, hi = 4.0 * hb - 2.0 * hb, 4.0 * hb + 2.0 * hb
    iv = [lo + 0.4 * (hi - lo), lo + 0.45 * (hi - lo), lo, hi]
    v = O.seeded_normal(n, 12)
    y_ref = O.cheb_av(O.find_pol(iv, max_deg=80), ia, ja, a, v)
    try:
        for variant in range(7):
            gpu_lib.set_filter_kernel(variant)
            gpu_lib.set_csr(ia, ja, a)
            assert 0 < gpu_lib.row_pattern_count() <= 1024
            pol = gpu_lib.find_pol(iv, max_deg=80)
            if variant not in (0, 3):
                with pytest.raises(Exception, match="not available"):
                    gpu_lib.chebav(pol, v)
            else:
                assert np.array_equal(gpu_lib.chebav(pol, v), y_ref), variant
            gpu_lib.free_pol(pol)
    finally:
        gpu_lib.set_filter_kernel(-1)


@pytest.mark.parametrize("dims, M, nvec", [((30, 30, 30), 300, 30), ((100, 100, 1), 500, 30), ((17, 13, 11), 7, 30),
                                           ((20, 20, 20), 60, 64), ((20, 20, 20), 61, 45)])
def test_kpm_product_identities_match_direct_dots(gpu_lib, dims, M, nvec):
    """KPM moments from the Chebyshev product identities (two moments per
    block product) agree with the direct per-degree dots with the probes
    within the moment bar (1e-12 of ||mu||_inf): odd and even moment counts,
    and more than 32 probes (several 32-probe launches per step, with paired
    16-byte loads for an even count and single loads for an odd one)."""
    ia, ja, a = _lap(gpu_lib, *dims)
    n = len(ia) - 1
    hi = 12.0 if dims[2] > 1 else 8.0
    probes = O.seeded_normal(n * nvec, 77).reshape(nvec, n)
    try:
        out = {}
        for dbl in (1, 0):
            gpu_lib.lib.evslcu_set_kpm_doubling(dbl)
            out[dbl] = gpu_lib.kpmdos_probes(M, 1, probes, [0.6, 1.2, 0.0, hi])
        mu1, ec1 = out[1]
        mu0, ec0 = out[0]
        assert np.max(np.abs(mu1 - mu0)) <= 1e-12 * np.max(np.abs(mu0))
        assert abs(ec1 - ec0) <= 1e-10 * max(abs(ec0), 1.0)
    finally:
        gpu_lib.lib.evslcu_set_kpm_doubling(1)


def _lap9_csr(nx, ny):
    """2-D 9-point stencil (8 on the diagonal, -1 to the 8 neighbours)."""
    rows = []
    for j in range(ny):
        for i in range(nx):
            cols, vals = [], []
            for dj in (-1, 0, 1):
                for di in (-1, 0, 1):
                    ii, jj = i + di, j + dj
                    if 0 <= ii < nx and 0 <= jj < ny:
                        cols.append(jj * nx + ii)
                        vals.append(8.0 if (di == 0 and dj == 0) else -1.0)
            rows.append((cols, vals))
    return _csr_from_rows(rows)


@pytest.mark.parametrize("variant", range(7))
def test_filter_kernels_on_nine_entry_rows(gpu_lib, variant):
    """Rows of 9 stored entries take the 16-wide unrolled row products
    (variants 1, 2 and 5) and every other form: each gives the reference's
    filtered vector bit for bit."""
    ia, ja, a = _lap9_csr(61, 47)
    n = len(ia) - 1
    gpu_lib.set_filter_kernel(variant)
    try:
        gpu_lib.set_csr(ia, ja, a)
        assert gpu_lib.row_pattern_count() == 9
        iv = [3.0, 4.0, -1.0, 17.0]
        v = O.seeded_normal(n, 21)
        pol = gpu_lib.find_pol(iv, max_deg=120)
        y = gpu_lib.chebav(pol, v)
        gpu_lib.free_pol(pol)
        y_ref = O.cheb_av(O.find_pol(iv, max_deg=120), ia, ja, a, v)
        assert np.array_equal(y, y_ref), (variant, np.max(np.abs(y - y_ref)))
        assert np.array_equal(gpu_lib.matvec(v), O.csr_matvec(ia, ja, a, v))
    finally:
        gpu_lib.set_filter_kernel(-1)


@pytest.mark.parametrize("nvec", [20, 13])
def test_kpm_prefetch_form_is_bitwise(gpu_lib, nvec):
    """The KPM block step that loads each row's own v_k, v_k-1 before its
    gathers (and stores 16 bytes at a time) performs the same operations:
    its raw dot products equal the default form's bit for bit, even and odd
    probe counts (paired and single loads)."""
    import evsl_b200

    ia, ja, a = _lap(gpu_lib, 14, 12, 5)
    n = len(ia) - 1
    iv = [0.7, 2.9, 0.0, 12.0]
    probes = evsl_b200.DeviceBuffer.from_host(gpu_lib.lib, O.seeded_rademacher(nvec, n, 5))
    ref = gpu_lib.kpm_dots(40, iv, probes, nvec)
    try:
        gpu_lib.lib.evslcu_set_kpm_prefetch(1)
        got = gpu_lib.kpm_dots(40, iv, probes, nvec)
    finally:
        gpu_lib.lib.evslcu_set_kpm_prefetch(0)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("case", ["lap3d", "rspd"])
def test_matvec_cols_bitwise(gpu_lib, case):
    """The block matvec the Ritz residuals use (all columns in one launch)
    equals the reference CPU CSR matvec (SRC/spmat.c:257-298) column by
    column bit for bit: on the row-pattern dictionary of a Laplacian and on
    the SELL-C-sigma copy of a random SPD matrix."""
    from evsl_b200 import workloads as W

    ia, ja, a = O.lap_csr(23, 19, 17) if case == "lap3d" else W.random_spd_csr(7001, 16, 41)
    gpu_lib.set_csr(ia, ja, a)
    n = len(ia) - 1
    X = np.stack([O.seeded_normal(n, 60 + c) for c in range(37)])
    Y = gpu_lib.matvec_cols(X)
    for c in range(X.shape[0]):
        assert np.array_equal(Y[c], O.csr_matvec(ia, ja, a, X[c])), c
