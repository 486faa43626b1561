"""The C-ABI library loads and exports every function include/*.h declares,
and its host-only entry points (filter design, slicing, damping) reproduce
the reference bit for bit without touching a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import evsl_b200
from oracle import evsl_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROTO = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*\**\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(", re.M)


def declared_functions():
    names = set()
    for h in ("evsl.h", "evslx.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"#define[^\n]*(\\\n[^\n]*)*", "", text)
        text = re.sub(r"typedef[^;]*;", "", text)
        for m in PROTO.finditer(text):
            name = m.group(1)
            if name in ("if", "while", "for", "return", "sizeof", "typedef"):
                continue
            names.add(name)
    return sorted(names)


def test_library_loads():
    lib = evsl_b200.load()
    assert os.path.exists(evsl_b200.library_path())
    assert lib is not None


def test_every_declared_symbol_is_exported():
    lib = evsl_b200.load()
    names = declared_functions()
    assert "ChebLanNr" in names and "kpmdos" in names and "evslx_kpmdos_probes" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def _find_pol(lib, iv, damping, ti, te, md):
    pol = evsl_b200.PolParams()
    lib.set_pol_def(C.byref(pol))
    pol.damping, pol.thresh_int, pol.thresh_ext, pol.max_deg = damping, ti, te, md
    arr = np.ascontiguousarray(iv, dtype=np.float64)
    rc = lib.find_pol(arr.ctypes.data_as(C.POINTER(C.c_double)), C.byref(pol))
    return rc, pol


def test_find_pol_matches_reference_bitwise(golden):
    lib = evsl_b200.load()
    i = 0
    while f"fp{i}_intv" in golden:
        damp, ti, te, md = golden[f"fp{i}_cfg"]
        rc, pol = _find_pol(lib, list(golden[f"fp{i}_intv"]), int(damp), ti, te, int(md))
        assert rc == 0
        d = pol.as_dict()
        typ, deg, cc, dd, gam, bar = golden[f"fp{i}_scal"]
        assert (d["type"], d["deg"]) == (typ, deg), i
        assert (d["cc"], d["dd"], d["gam"], d["bar"]) == (cc, dd, gam, bar), i
        assert np.array_equal(d["mu"], golden[f"fp{i}_mu"]), i
        lib.free_pol(C.byref(pol))
        i += 1


def test_find_pol_rejects_bad_interval():
    lib = evsl_b200.load()
    for iv in ([1.0, 0.5, 0.0, 8.0], [9.0, 10.0, 0.0, 8.0], [-3.0, -1.0, 0.0, 8.0]):
        rc, pol = _find_pol(lib, iv, 2, 0.8, 0.2, 3000)
        assert rc == -1


def test_spslicer_matches_reference_bitwise(golden):
    lib = evsl_b200.load()
    for key, mukey, ekey, iv, nint in (("sli20", "kpm20_mu", "kpm20_ecnt", [0.6, 1.2, 0.0, 8.0], 4),
                                       ("sli8", "kpm8_mu", "kpm8_ecnt", [0.6, 2.0, 0.0, 12.0], 5)):
        mu = np.ascontiguousarray(golden[mukey])
        sli = np.zeros(nint + 1)
        iva = np.ascontiguousarray(iv, dtype=np.float64)
        dp = C.POINTER(C.c_double)
        rc = lib.spslicer(sli.ctypes.data_as(dp), mu.ctypes.data_as(dp), len(mu) - 1, iva.ctypes.data_as(dp),
                          nint, int(10 * golden[ekey][0]))
        assert rc == 0
        assert np.array_equal(sli, golden[key])


def test_spslicer_edge_cases():
    lib = evsl_b200.load()
    dp = C.POINTER(C.c_double)
    mu = np.ascontiguousarray(O.dampcf(30, 1))
    # single slice returns the interval itself
    sli = np.zeros(2)
    iv = np.array([0.6, 1.2, 0.0, 8.0])
    assert lib.spslicer(sli.ctypes.data_as(dp), mu.ctypes.data_as(dp), 30, iv.ctypes.data_as(dp), 1, 10) == 0
    assert list(sli) == [0.6, 1.2]
    bad = np.array([1.2, 0.6, 0.0, 8.0])
    assert lib.spslicer(sli.ctypes.data_as(dp), mu.ctypes.data_as(dp), 30, bad.ctypes.data_as(dp), 2, 10) == -1


def test_dampcf_matches_restatement():
    lib = evsl_b200.load()
    for m in (5, 40, 300):
        for damping in (0, 1, 2):
            jac = np.zeros(m + 1)
            lib.dampcf(m, damping, jac.ctypes.data_as(C.POINTER(C.c_double)))
            assert np.array_equal(jac, O.dampcf(m, damping)), (m, damping)


def test_start_fails_loudly_without_gpu():
    lib = evsl_b200.load()
    from evsl_b200 import EvslError

    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(EvslError):
        evsl_b200.Library()


@pytest.mark.parametrize("k, m, kind", [(3000, 1500, "random"), (3000, 1500, "repeated"), (200, 50, "random")])
def test_tridiagonal_eigenvectors_host(k, m, kind):
    """Inverse iteration for the Ritz step's tridiagonal eigenvectors (host,
    split over threads at cluster starts when the work is large): each
    vector solves T z = lambda z to 1e-12 of ||T||, the vectors are
    orthonormal to 1e-12 (also inside clusters of exactly repeated
    eigenvalues, where only the span is defined), and a second call gives
    the same bits.  3000 x 1500 runs on two threads."""
    lib = evsl_b200.load()
    vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    lib.evsl_trid_eigvecs.restype = C.c_int
    lib.evsl_trid_eigvecs.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
    lib.evsl_trid_eigvals.restype = C.c_int
    lib.evsl_trid_eigvals.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(k + m)
    if kind == "random":
        d, e = rng.uniform(-0.1, 1.0, k), rng.uniform(0.01, 0.3, k - 1)
    else:  # four identical blocks: every eigenvalue four times
        b = k // 4
        d = np.tile(rng.uniform(-0.1, 1.0, b), 4)
        e = np.tile(np.r_[rng.uniform(0.01, 0.3, b - 1), 0.0], 4)[: k - 1]
    w = np.zeros(k)
    assert lib.evsl_trid_eigvals(k, vp(d), vp(e), vp(w)) == 0
    sel = np.ascontiguousarray(w[-m:])
    Z = np.zeros((m, k))
    assert lib.evsl_trid_eigvecs(k, vp(d), vp(e), m, vp(sel), vp(Z), k) == 0
    Z2 = np.zeros((m, k))
    assert lib.evsl_trid_eigvecs(k, vp(d), vp(e), m, vp(sel), vp(Z2), k) == 0
    assert np.array_equal(Z, Z2)
    tn = np.max(np.abs(d) + np.r_[np.abs(e), 0] + np.r_[0, np.abs(e)])
    TZ = d * Z + np.c_[Z[:, 1:] * e, np.zeros(m)] + np.c_[np.zeros(m), Z[:, :-1] * e]
    assert np.max(np.abs(TZ - sel[:, None] * Z)) <= 1e-12 * tn
    assert np.max(np.abs(Z @ Z.T - np.eye(m))) <= 1e-12


@pytest.mark.skipif(not os.path.exists(O.REF_LIB_PATH), reason="reference build oracle/_ref not present")
def test_find_pol_threaded_search_matches_reference_bitwise():
    """The library's filter design on narrow mid-spectrum intervals, where
    the degree search runs over host threads (starting degree >= 100),
    designed and forced degrees and all three dampings: degree, type,
    coefficients, gam and bar equal the reference build's bit for bit."""
    lib = evsl_b200.load()
    R = O.RefLib()
    rng = np.random.default_rng(23)
    for i in range(18):
        lo, hi = 0.0, 12.0 + rng.uniform()
        c = lo + rng.uniform(0.1, 0.9) * (hi - lo)
        w = (hi - lo) * 10.0 ** rng.uniform(-4.0, -2.5)
        iv = [c - w / 2, c + w / 2, lo, hi]
        damping = i % 3
        # start of the design loop: 2 + 0.5 / (width in [-1, 1])
        dmin = int(2 + 0.5 / (w / ((hi - lo) / 2))) + 1
        forced = 0 if i % 2 else int(rng.integers(dmin, dmin + 300))
        rc_r, pol_r = R.find_pol(iv, damping=damping, thresh_int=0.8, thresh_ext=0.2, max_deg=6000, deg=forced)
        ref = R.pol_dict(pol_r)
        R.free_pol(pol_r)
        pol = evsl_b200.PolParams()
        lib.set_pol_def(C.byref(pol))
        pol.damping, pol.thresh_int, pol.thresh_ext, pol.max_deg, pol.deg = damping, 0.8, 0.2, 6000, forced
        arr = np.ascontiguousarray(iv, dtype=np.float64)
        rc = lib.find_pol(arr.ctypes.data_as(C.POINTER(C.c_double)), C.byref(pol))
        assert rc == rc_r == 0, (i, iv)
        assert pol.deg == ref["deg"] and pol.type == ref["type"], (i, iv, forced, pol.deg, ref["deg"])
        mu = np.ctypeslib.as_array(pol.mu, (pol.deg + 1,)).copy()
        assert np.array_equal(mu, ref["mu"]), (i, iv, forced)
        assert pol.gam == ref["gam"] and pol.bar == ref["bar"], (i, iv, forced)
        lib.free_pol(C.byref(pol))
