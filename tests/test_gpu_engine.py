"""GPU tests of the multi-column filter, the mixed-precision path and the
request engine (batched and served slice solves, DOS requests).

Tolerances (written per test):
  * FP64 multi-column filter: every column bitwise equal to ChebAv;
  * FP32 multi-column filter: ||y32 - y64|| <= 1e-4 ||y64|| per column;
  * FP64 engine vs ChebLanNr: counts equal, eigenvalues within 1e-10 x
    (spectral width), residuals < tol;
  * mixed precision after FP64 refinement: counts exact against the
    analytic (or dense) spectrum, eigenvalues within 1e-8 x (spectral
    width), residuals < tol;
  * a request alone and in a mix of requests: bitwise equal results;
  * engine DOS request vs kpmdos with the same generator seed: bitwise.
"""
import numpy as np
import pytest

import evsl_b200 as E
from evsl_b200 import workloads as W
from oracle import evsl_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def mixed_on_small(gpu_lib):
    """These tests check the mixed-precision path on small matrices, which
    the engine would otherwise filter in FP64."""
    gpu_lib.set_mixed_min_rows(0)
    yield
    gpu_lib.set_mixed_min_rows(131072)


def _pols(lib, intvs, **kw):
    return [lib.find_pol(iv, **kw) for iv in intvs]


def test_multi_filter_fp64_bitwise_fp32_close(gpu_lib):
    cases = [(O.lap_csr(41, 53, 1), 8.0), (O.lap_csr(20, 20, 20), 12.0), (W.random_spd_csr(6000, 16, 2), None)]
    for (ia, ja, a), hi in cases:
        gpu_lib.set_csr(ia, ja, a)
        n = len(ia) - 1
        if hi is None:
            lo_b, hi_b = W.gershgorin_bounds(ia, ja, a)
            lo_b = max(lo_b, 0.0)
        else:
            lo_b, hi_b = 0.0, hi
        w = hi_b - lo_b
        intvs = [[lo_b + f0 * w, lo_b + f1 * w, lo_b, hi_b] for f0, f1 in
                 ((0.05, 0.1), (0.2, 0.22), (0.3, 0.5), (0.6, 0.61), (0.0, 0.03), (0.9, 1.0))]
        pols = _pols(gpu_lib, intvs, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=400)
        X = O.seeded_normal(n * len(pols), 4).reshape(len(pols), n)
        Y64 = gpu_lib.chebav_multi(pols, X, E.PREC_FP64)
        Y32 = gpu_lib.chebav_multi(pols, X, E.PREC_MIXED)
        for c, pol in enumerate(pols):
            ref = gpu_lib.chebav(pol, X[c])
            assert np.array_equal(Y64[c], ref)
            assert np.linalg.norm(Y32[c] - ref) <= 1e-4 * np.linalg.norm(ref)
        for p in pols:
            gpu_lib.free_pol(p)


def test_filter_variants_and_autotuner(gpu_lib):
    """All kernel variants (SELL-32 and row-pattern dictionary) give the same
    bits; the autotuner picks one; a dictionary variant forced on a matrix
    without a dictionary fails with an error."""
    ia, ja, a = O.lap_csr(40, 40, 40)
    gpu_lib.set_csr(ia, ja, a)
    assert gpu_lib.row_pattern_count() == 27
    n = len(ia) - 1
    pol = gpu_lib.find_pol([0.6, 0.9, 0.0, 12.0])
    try:
        for prec in (E.PREC_FP64, E.PREC_MIXED):
            for B in (1, 3, 8, 16):
                X = O.seeded_normal(n * B, 30 + B).reshape(B, n)
                gpu_lib.set_filter_variant(-1)
                ref = gpu_lib.chebav_multi([pol] * B, X, prec)
                assert 0 <= gpu_lib.tuned_filter_variant(prec, B) <= 5
                for v in range(6):
                    gpu_lib.set_filter_variant(v)
                    assert np.array_equal(gpu_lib.chebav_multi([pol] * B, X, prec), ref), (prec, B, v)
        ia, ja, a = W.random_spd_csr(3000, 8, 5)
        gpu_lib.set_csr(ia, ja, a)
        assert gpu_lib.row_pattern_count() == 0
        lo, hi = W.gershgorin_bounds(ia, ja, a)
        pol2 = gpu_lib.find_pol([lo + 0.3 * (hi - lo), lo + 0.4 * (hi - lo), lo, hi], max_deg=50)
        gpu_lib.set_filter_variant(4)
        with pytest.raises(Exception, match="dictionary"):
            gpu_lib.chebav_multi([pol2] * 2, O.seeded_normal(6000, 3).reshape(2, 3000), E.PREC_FP64)
        gpu_lib.free_pol(pol2)
    finally:
        gpu_lib.set_filter_variant(-1)
        gpu_lib.free_pol(pol)


def _lap_slices(ev, starts, count):
    out = []
    for s in starts:
        a, b, cnt = W.gap_interval(ev, s, count)
        out.append(([a, b], cnt))
    return out


def test_engine_fp64_matches_cheblan_nr(gpu_lib):
    ia, ja, a = O.lap_csr(100, 100, 1)
    gpu_lib.set_csr(ia, ja, a)
    ev = W.laplacian_eigenvalues(100, 100, 1)
    sl = _lap_slices(ev, (0.6, 0.75, 0.9), 40)
    intvs = [[x[0][0], x[0][1], 0.0, 8.0] for x in sl]
    pols = _pols(gpu_lib, intvs)
    v = O.seeded_normal(10000, 1234)
    batch = gpu_lib.cheblan_nr_batch(intvs, 2000, 1e-8, v, pols, E.PREC_FP64)
    for s, (lam_b, Y_b, res_b) in enumerate(batch):
        lam, Y, res = gpu_lib.cheblan_nr(intvs[s], 2000, 1e-8, v, pols[s], want_vectors=False)
        exact = ev[(ev >= intvs[s][0]) & (ev <= intvs[s][1])]
        assert len(lam_b) == len(lam) == len(exact) == sl[s][1]
        assert np.max(np.abs(np.sort(lam_b) - np.sort(lam))) <= 1e-10 * 8.0
        assert np.all(res_b < 1e-8)
        G = Y_b @ Y_b.T
        assert np.max(np.abs(G - np.eye(len(lam_b)))) < 1e-8
    for p in pols:
        gpu_lib.free_pol(p)


def test_engine_mixed_precision_accuracy(gpu_lib):
    """3-D Laplacian 30^3: FP32 filter + FP64 refinement meets tol 1e-8."""
    ia, ja, a = O.lap_csr(30, 30, 30)
    gpu_lib.set_csr(ia, ja, a)
    ev = W.laplacian_eigenvalues(30, 30, 30)
    sl = _lap_slices(ev, (0.6, 1.0), 50)
    intvs = [[x[0][0], x[0][1], 0.0, 12.0] for x in sl]
    pols = _pols(gpu_lib, intvs)
    v = O.seeded_normal(27000, 9)
    batch = gpu_lib.cheblan_nr_batch(intvs, 1500, 1e-8, v, pols, E.PREC_MIXED)
    for s, (lam, Y, res) in enumerate(batch):
        exact = ev[(ev >= intvs[s][0]) & (ev <= intvs[s][1])]
        assert len(lam) == len(exact) == sl[s][1]
        assert np.max(np.abs(np.sort(lam) - exact)) <= 1e-8 * 12.0
        assert np.all(res < 1e-8)
    for p in pols:
        gpu_lib.free_pol(p)


@pytest.mark.parametrize("precision", [E.PREC_FP64, E.PREC_MIXED])
def test_engine_request_same_alone_and_in_mix(gpu_lib, precision):
    ia, ja, a = O.lap_csr(60, 60, 1)
    ia2, ja2, a2 = O.lap_csr(18, 17, 16)
    ev = W.laplacian_eigenvalues(60, 60, 1)
    ev2 = W.laplacian_eigenvalues(18, 17, 16)
    gpu_lib.set_csr(ia, ja, a)
    M1 = gpu_lib.matrix(ia, ja, a)
    M2 = gpu_lib.matrix(ia2, ja2, a2)
    (i1, c1), (i2, c2) = _lap_slices(ev, (0.5, 1.1), 30)
    (i3, c3), = _lap_slices(ev2, (0.8,), 25)
    iv1, iv2, iv3 = [i1[0], i1[1], 0.0, 8.0], [i2[0], i2[1], 0.0, 8.0], [i3[0], i3[1], 0.0, 12.0]
    p1, p2, p3 = gpu_lib.find_pol(iv1), gpu_lib.find_pol(iv2), gpu_lib.find_pol(iv3)
    v1 = O.seeded_normal(3600, 1)
    v3 = O.seeded_normal(len(ia2) - 1, 3)

    eng = gpu_lib.engine(4, precision=precision)
    eng.submit_slice(M1, iv1, p1, 1000, 1e-8, v1, 7)
    eng.run()
    alone = eng.pop()
    # one column: FP64 runs the single-vector filter, mixed a captured graph
    assert eng.group_widths()[1] > 0
    assert (eng.plan_builds() >= 1) == (precision == E.PREC_MIXED)
    eng.free()
    # the same request with the filters launched directly (no captured graphs)
    eng = gpu_lib.engine(4, precision=precision)
    eng.use_graphs(False)
    eng.submit_slice(M1, iv1, p1, 1000, 1e-8, v1, 7)
    eng.run()
    direct = eng.pop()
    eng.free()
    assert np.array_equal(alone["lam"], direct["lam"]) and np.array_equal(alone["res"], direct["res"])

    eng = gpu_lib.engine(4, precision=precision)
    eng.submit_slice(M1, iv2, p2, 1000, 1e-8, v1, 1)
    eng.submit_kpm(M2, 60, 1, 8, iv3, 5, 2)
    eng.submit_slice(M2, iv3, p3, 1000, 1e-8, v3, 3)
    eng.step()
    eng.step()
    eng.submit_slice(M1, iv1, p1, 1000, 1e-8, v1, 7)  # joins while the others run
    eng.run()
    got = {}
    while True:
        r = eng.pop()
        if r is None:
            break
        got[r["tag"]] = r
    eng.free()
    mixed = got[7]
    assert alone["rc"] == 0 and mixed["rc"] == 0
    assert alone["nev"] == mixed["nev"] == c1
    assert np.array_equal(alone["lam"], mixed["lam"]) and np.array_equal(alone["res"], mixed["res"])
    assert got[1]["nev"] == c2 and got[3]["nev"] == c3
    for r in (got[1], got[3], mixed):
        assert np.all(r["res"] < 1e-8)
    M1.free()
    M2.free()
    for p in (p1, p2, p3):
        gpu_lib.free_pol(p)


def test_engine_kpm_equals_kpmdos(gpu_lib):
    ia, ja, a = O.lap_csr(30, 30, 12)
    gpu_lib.set_csr(ia, ja, a)
    M = gpu_lib.matrix(ia, ja, a)
    iv = [0.6, 2.0, 0.0, 12.0]
    eng = gpu_lib.engine(2)
    eng.submit_kpm(M, 80, 1, 70, iv, 1234, 11)
    eng.run()
    r = eng.pop()
    eng.free()
    gpu_lib.set_seed(1234)
    mu, ec = gpu_lib.kpmdos(80, 1, 70, iv)
    assert r["rc"] == 0 and np.array_equal(r["mu"], mu) and r["ecnt"] == ec
    M.free()


def test_engine_hbm_budget_admission(gpu_lib):
    ia, ja, a = O.lap_csr(50, 50, 1)
    gpu_lib.set_csr(ia, ja, a)
    M = gpu_lib.matrix(ia, ja, a)
    ev = W.laplacian_eigenvalues(50, 50, 1)
    sl = _lap_slices(ev, (0.5, 0.9, 1.3), 20)
    intvs = [[x[0][0], x[0][1], 0.0, 8.0] for x in sl]
    pols = _pols(gpu_lib, intvs)
    v = O.seeded_normal(2500, 2)
    maxit = 600
    # device bytes the engine reserves for one request (basis, start and
    # restart vectors, Gram-Schmidt workspace); the budget admits one at a time
    req = 8 * (2500 * (maxit + 3) + ((2500 + 1023) // 1024) * (maxit + 1) + (maxit + 1) + 8)
    one = int(1.5 * req)
    results = []
    for budget in (0, one):
        eng = gpu_lib.engine(3, hbm_budget=budget)
        for s, iv in enumerate(intvs):
            eng.submit_slice(M, iv, pols[s], maxit, 1e-8, v, s)
        peak = 0
        while eng.step() > 0:
            peak = max(peak, eng.bytes_in_use())
            if budget:
                assert eng.bytes_in_use() <= budget
        out = {}
        while True:
            r = eng.pop()
            if r is None:
                break
            out[r["tag"]] = r
        results.append(out)
        eng.free()
        if budget:
            assert req <= peak <= budget
    for s in range(3):
        assert results[0][s]["nev"] == results[1][s]["nev"] == sl[s][1]
        assert np.array_equal(results[0][s]["lam"], results[1][s]["lam"])
    # a request larger than the whole budget fails instead of blocking
    eng = gpu_lib.engine(2, hbm_budget=1 << 20)
    eng.submit_slice(M, intvs[0], pols[0], maxit, 1e-8, v, 99)
    eng.run()
    r = eng.pop()
    assert r["tag"] == 99 and r["rc"] != 0
    eng.free()
    M.free()
    for p in pols:
        gpu_lib.free_pol(p)


def test_mixed_precision_random_spd(gpu_lib):
    """The random sparse SPD family of the mixed-precision workload at a size
    the dense solver checks: a slice of ~30 eigenvalues in the lower
    interior, FP32 filter + FP64 refinement."""
    n = 4000
    ia, ja, a = W.random_spd_csr(n, 16, 21)
    gpu_lib.set_csr(ia, ja, a)
    M = np.zeros((n, n))
    for i in range(n):
        M[i, ja[ia[i]:ia[i + 1]]] = a[ia[i]:ia[i + 1]]
    ev = np.linalg.eigvalsh(M)
    v = O.seeded_normal(n, 5)
    lo, hi = gpu_lib.lan_trbounds(50, 200, 1e-8, v, 1)
    a0, b0, cnt = W.gap_interval(ev, ev[n // 4], 30)
    iv = [a0, b0, lo, hi]
    pol = gpu_lib.find_pol(iv)
    (lam64, _, res64), = gpu_lib.cheblan_nr_batch([iv], 2000, 1e-8, v, [pol], E.PREC_FP64, want_vectors=False)
    (lam32, _, res32), = gpu_lib.cheblan_nr_batch([iv], 2000, 1e-8, v, [pol], E.PREC_MIXED, want_vectors=False)
    exact = ev[(ev >= a0) & (ev <= b0)]
    width = hi - lo
    assert len(lam64) == len(lam32) == len(exact) == cnt
    assert np.max(np.abs(np.sort(lam64) - exact)) <= 1e-10 * width
    assert np.max(np.abs(np.sort(lam32) - exact)) <= 1e-8 * width
    assert np.all(res64 < 1e-8) and np.all(res32 < 1e-8)
    gpu_lib.free_pol(pol)


@pytest.mark.parametrize("precision", [E.PREC_FP64, E.PREC_MIXED])
def test_engine_many_uneven_instances(gpu_lib, precision):
    """Batched uneven instances: 12 independent 2-D/3-D Laplacians with n
    log-uniform in [1e3, 3e4] (sizes from a seed), each with its own interval
    of 20-60 eigenvalues and its own filter degree, all in one engine."""
    rng = np.random.default_rng(4)
    eng = gpu_lib.engine(12, precision=precision)
    mats, expect, pols = [], {}, []
    for i in range(12):
        nn = int(np.exp(rng.uniform(np.log(1e3), np.log(3e4))))
        if i % 2 == 0:
            s = max(int(round(np.sqrt(nn))), 10)
            dims, hi = (s, s + i % 3, 1), 8.0
        else:
            s = max(int(round(nn ** (1 / 3))), 8)
            dims, hi = (s, s + 1, s), 12.0
        ia, ja, a = O.lap_csr(*dims)
        ev = np.sort(W.laplacian_eigenvalues(*dims))
        a0, b0, cnt = W.gap_interval(ev, float(rng.uniform(0.3, 1.5)), int(rng.integers(20, 61)))
        iv = [a0, b0, 0.0, hi]
        M = gpu_lib.matrix(ia, ja, a)
        pol = gpu_lib.find_pol(iv)
        mats.append(M)
        pols.append(pol)
        expect[i] = ev[(ev >= a0) & (ev <= b0)]
        eng.submit_slice(M, iv, pol, 2000, 1e-8, O.seeded_normal(len(ia) - 1, i), i)
    eng.run()
    n_done = 0
    while True:
        r = eng.pop()
        if r is None:
            break
        ex = expect[r["tag"]]
        assert r["rc"] == 0 and r["nev"] == len(ex)
        width = 8.0 if r["tag"] % 2 == 0 else 12.0
        tol_eig = (1e-10 if precision == E.PREC_FP64 else 1e-8) * width
        assert np.max(np.abs(np.sort(r["lam"]) - ex)) <= tol_eig
        assert np.all(r["res"] < 1e-8)
        n_done += 1
    assert n_done == 12
    eng.free()
    for M in mats:
        M.free()
    for p in pols:
        gpu_lib.free_pol(p)


def test_mixed_engine_filters_small_matrices_in_fp64(gpu_lib):
    """With the default threshold a mixed engine runs small matrices in
    FP64: the result equals the FP64 engine's bit for bit."""
    gpu_lib.set_mixed_min_rows(131072)
    ia, ja, a = O.lap_csr(40, 40, 1)
    gpu_lib.set_csr(ia, ja, a)
    M = gpu_lib.matrix(ia, ja, a)
    iv = [0.7, 0.9, 0.0, 8.0]
    pol = gpu_lib.find_pol(iv)
    v = O.seeded_normal(1600, 3)
    out = []
    for prec in (E.PREC_FP64, E.PREC_MIXED):
        eng = gpu_lib.engine(2, precision=prec)
        eng.submit_slice(M, iv, pol, 1000, 1e-8, v, 1)
        eng.run()
        out.append(eng.pop())
        eng.free()
    assert out[0]["nev"] == out[1]["nev"] > 0 and out[1]["refine_sweeps"] == 0
    assert np.array_equal(out[0]["lam"], out[1]["lam"])
    M.free()
    gpu_lib.free_pol(pol)


def test_multi_filter_dictionary_with_double_table(gpu_lib):
    """The multi-column dictionary kernels (variants 4, 5) on a table that
    holds doubles (a diagonal shifted by 1e-9 every 7th row, so the values
    are not floats): every variant gives the same bits as variant 0, in FP64
    and FP32, and FP64 matches ChebAv column by column."""
    ia, ja, a = O.lap_csr(22, 19, 17)
    a = a.copy()
    n = len(ia) - 1
    for r in range(0, n, 7):
        for j in range(ia[r], ia[r + 1]):
            if ja[j] == r:
                a[j] += 1e-9
    gpu_lib.set_csr(ia, ja, a)
    assert 0 < gpu_lib.row_pattern_count() <= 1024
    pol = gpu_lib.find_pol([0.6, 0.9, 0.0, 12.0], max_deg=200)
    try:
        for prec in (E.PREC_FP64, E.PREC_MIXED):
            for B in (1, 4, 16):
                X = O.seeded_normal(n * B, 40 + B).reshape(B, n)
                gpu_lib.set_filter_variant(0)
                ref = gpu_lib.chebav_multi([pol] * B, X, prec)
                for v in (1, 2, 3, 4, 5):
                    gpu_lib.set_filter_variant(v)
                    assert np.array_equal(gpu_lib.chebav_multi([pol] * B, X, prec), ref), (prec, B, v)
                if prec == E.PREC_FP64:
                    gpu_lib.set_filter_variant(-1)
                    for c in range(B):
                        assert np.array_equal(ref[c], gpu_lib.chebav(pol, X[c]))
    finally:
        gpu_lib.set_filter_variant(-1)
        gpu_lib.free_pol(pol)


@pytest.mark.parametrize("persistent", [False, True])
def test_engine_batched_filter_is_bitwise_the_per_matrix_filter(gpu_lib, persistent):
    """The engine's batched filter (the lone FP64 columns of all small
    matrices advanced one degree per launch together, or all degrees in one
    persistent launch) gives every instance the same eigenvalues, bit for
    bit, as filtering each matrix on its own."""
    rng = np.random.default_rng(8)
    mats, pols, subs = [], [], []
    for i in range(10):
        nn = int(np.exp(rng.uniform(np.log(500), np.log(2e4))))
        if i % 2 == 0:
            s = max(int(round(np.sqrt(nn))), 10)
            dims, hi = (s, s + 1, 1), 8.0
        else:
            s = max(int(round(nn ** (1 / 3))), 8)
            dims, hi = (s, s, s + 1), 12.0
        ia, ja, a = O.lap_csr(*dims)
        ev = np.sort(W.laplacian_eigenvalues(*dims))
        a0, b0, cnt = W.gap_interval(ev, float(rng.uniform(0.4, 1.2)), int(rng.integers(15, 40)))
        iv = [a0, b0, 0.0, hi]
        M = gpu_lib.matrix(ia, ja, a)
        pol = gpu_lib.find_pol(iv)
        mats.append(M)
        pols.append(pol)
        subs.append((M, iv, pol, O.seeded_normal(len(ia) - 1, 30 + i), i, len(ev[(ev >= a0) & (ev <= b0)])))
    out = {}
    for batch in (True, False):
        eng = gpu_lib.engine(len(subs), precision=E.PREC_FP64)
        eng.use_batch(batch)
        gpu_lib.set_batch_persistent(persistent)
        for M, iv, pol, v, tag, _ in subs:
            eng.submit_slice(M, iv, pol, 1500, 1e-8, v, tag)
        try:
            eng.run()
        finally:
            gpu_lib.set_batch_persistent(False)
        res = {}
        while True:
            r = eng.pop()
            if r is None:
                break
            res[r["tag"]] = r
        assert (eng.batched_columns() > 0) == batch
        eng.free()
        out[batch] = res
    for _, _, _, _, tag, cnt in subs:
        a, b = out[True][tag], out[False][tag]
        assert a["rc"] == b["rc"] == 0 and a["nev"] == b["nev"] == cnt
        assert np.array_equal(a["lam"], b["lam"]) and np.array_equal(a["res"], b["res"])
    for M in mats:
        M.free()
    for p in pols:
        gpu_lib.free_pol(p)


def test_engine_batched_uneven_instances_full_scale(gpu_lib, persistent=False):
    """The batched-instances configuration at full scale: 128 independent
    2-D / 3-D Laplacians, n log-uniform in [1e3, 2e5] (4.85 million rows in
    all), each with its own interval of 20-80 eigenvalues (end points at gap
    midpoints) and its own find_pol degree, solved together by one FP64
    engine (the lone columns of all matrices filtered by the batched filter):
    every instance's count exact against its analytic spectrum, eigenvalues
    within 1e-10 x width, residuals < 1e-8."""
    import bench

    inst = bench.uneven_instances(128)
    gpu_lib.set_batch_persistent(persistent)
    eng = gpu_lib.engine(len(inst), precision=E.PREC_FP64)
    mats, pols = [], []
    for i, (dims, iv, _) in enumerate(inst):
        ia, ja, a = W.laplacian_csr(*dims)
        M = gpu_lib.matrix(ia, ja, a)
        gpu_lib.set_csr(ia, ja, a)
        pol = gpu_lib.find_pol(iv, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000)
        mats.append(M)
        pols.append(pol)
        eng.submit_slice(M, iv, pol, 1000, 1e-8, O.seeded_normal(len(ia) - 1, 100 + i), i)
    try:
        eng.run()
    finally:
        gpu_lib.set_batch_persistent(False)
    seen = 0
    while True:
        r = eng.pop()
        if r is None:
            break
        dims, iv, exact = inst[r["tag"]]
        assert r["rc"] == 0 and r["nev"] == len(exact), (r["tag"], dims, r["nev"], len(exact))
        assert np.max(np.abs(np.sort(r["lam"]) - exact)) <= 1e-10 * iv[3]
        assert np.all(r["res"] < 1e-8)
        seen += 1
    assert seen == len(inst) and eng.batched_columns() > 0
    eng.free()
    for M in mats:
        M.free()
    for p in pols:
        gpu_lib.free_pol(p)


def test_engine_persistent_batch_wait_times_out_and_recovers(gpu_lib):
    """Failure path of the persistent batched filter's dependency waits: with
    a limit of one poll a wait gives up, the engine step returns
    EVSLX_ERR_TIMEOUT (-105) with every block gone; with the default limit
    restored a new engine solves the same requests exactly."""
    rng = np.random.default_rng(9)
    subs, mats, pols = [], [], []
    for i in range(6):
        dims = (40 + 3 * i, 41, 1)
        ia, ja, a = O.lap_csr(*dims)
        ev = np.sort(W.laplacian_eigenvalues(*dims))
        a0, b0, cnt = W.gap_interval(ev, float(rng.uniform(0.5, 1.0)), 20)
        iv = [a0, b0, 0.0, 8.0]
        M = gpu_lib.matrix(ia, ja, a)
        pol = gpu_lib.find_pol(iv)
        mats.append(M)
        pols.append(pol)
        subs.append((M, iv, pol, O.seeded_normal(len(ia) - 1, 60 + i), i, len(ev[(ev >= a0) & (ev <= b0)])))
    gpu_lib.set_batch_persistent(True)
    try:
        gpu_lib.set_wait_limit(1)
        eng = gpu_lib.engine(len(subs), precision=E.PREC_FP64)
        for M, iv, pol, v, tag, _ in subs:
            eng.submit_slice(M, iv, pol, 1500, 1e-8, v, tag)
        with pytest.raises(E.EvslError) as err:
            eng.run()
        assert "returned -105" in str(err.value) and "ran out of polls" in gpu_lib.last_error()
        eng.free()
        gpu_lib.set_wait_limit(0)
        eng = gpu_lib.engine(len(subs), precision=E.PREC_FP64)
        for M, iv, pol, v, tag, _ in subs:
            eng.submit_slice(M, iv, pol, 1500, 1e-8, v, tag)
        eng.run()
        seen = 0
        while True:
            r = eng.pop()
            if r is None:
                break
            cnt = subs[r["tag"]][5]
            assert r["rc"] == 0 and r["nev"] == cnt and np.all(r["res"] < 1e-8)
            seen += 1
        assert seen == len(subs) and eng.batched_columns() > 0
        eng.free()
    finally:
        gpu_lib.set_wait_limit(0)
        gpu_lib.set_batch_persistent(False)
        for M in mats:
            M.free()
        for p in pols:
            gpu_lib.free_pol(p)


@pytest.mark.parametrize("precision", [E.PREC_FP64, E.PREC_MIXED])
def test_engine_batched_lanczos_ops_are_bitwise_per_slot(gpu_lib, precision):
    """The engine's Lanczos vector operations for all slots in one launch per
    operation (evslcu_lanczos_batch: every slot split into blocks as its own
    launches split it, reductions in the same order) give every request the
    same eigenvalues, residuals and step counts, bit for bit, as each slot's
    own launches -- with lone columns of several matrices, several slices of
    one matrix (multi-column groups) and the mixed-precision refinement."""
    rng = np.random.default_rng(12)
    mats, pols, subs = [], [], []
    specs = [((30, 31, 1), 8.0), ((14, 15, 16), 12.0), ((52, 50, 1), 8.0), ((70, 71, 1), 8.0)]
    for i, (dims, hi) in enumerate(specs):
        ia, ja, a = O.lap_csr(*dims)
        ev = np.sort(W.laplacian_eigenvalues(*dims))
        M = gpu_lib.matrix(ia, ja, a)
        mats.append(M)
        for j in range(2 if i == 3 else 1):
            a0, b0, cnt = W.gap_interval(ev, float(rng.uniform(0.4, 1.2)), int(rng.integers(12, 30)))
            iv = [a0, b0, 0.0, hi]
            pol = gpu_lib.find_pol(iv)
            pols.append(pol)
            subs.append((M, iv, pol, O.seeded_normal(len(ia) - 1, 80 + 10 * i + j), len(subs),
                         len(ev[(ev >= a0) & (ev <= b0)])))
    gpu_lib.set_mixed_min_rows(0)
    out = {}
    try:
        for batched in (True, False):
            eng = gpu_lib.engine(len(subs), precision=precision)
            eng.use_batch_ops(batched)
            for M, iv, pol, v, tag, _ in subs:
                eng.submit_slice(M, iv, pol, 1500, 1e-8, v, tag)
            eng.run()
            res = {}
            while True:
                r = eng.pop()
                if r is None:
                    break
                res[r["tag"]] = r
            eng.free()
            out[batched] = res
    finally:
        gpu_lib.set_mixed_min_rows(131072)
    for _, _, _, _, tag, cnt in subs:
        a, b = out[True][tag], out[False][tag]
        assert a["rc"] == b["rc"] == 0 and a["nev"] == b["nev"] == cnt
        assert a["lanczos_steps"] == b["lanczos_steps"]
        assert np.array_equal(a["lam"], b["lam"]) and np.array_equal(a["res"], b["res"])
    for M in mats:
        M.free()
    for p in pols:
        gpu_lib.free_pol(p)
