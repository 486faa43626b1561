"""The CPU oracle, pinned: the numpy restatement (oracle/evsl_oracle.py) against
the golden fixtures produced by the reference EVSL build, and -- where the
reference build is present -- against the reference library directly.

Tolerances: find_pol, ChebAv, spslicer and the Laplacian CSR are compared
bitwise (same floating-point operations); KPM moments normwise to 1e-13
(only the dot-product summation order differs); eigenvalues to 1e-12.
"""
import os

import numpy as np
import pytest

from oracle import evsl_oracle as O

HAVE_REF = os.path.exists(O.REF_LIB_PATH)


def _fp_cases(golden):
    i = 0
    while f"fp{i}_intv" in golden:
        yield i
        i += 1


def test_find_pol_restatement_matches_reference(golden):
    for i in _fp_cases(golden):
        iv = list(golden[f"fp{i}_intv"])
        damp, ti, te, md = golden[f"fp{i}_cfg"]
        p = O.find_pol(iv, damping=int(damp), thresh_int=ti, thresh_ext=te, max_deg=int(md))
        typ, deg, cc, dd, gam, bar = golden[f"fp{i}_scal"]
        assert p["type"] == typ and p["deg"] == deg, (i, p["type"], p["deg"], typ, deg)
        assert p["cc"] == cc and p["dd"] == dd and p["gam"] == gam and p["bar"] == bar, i
        assert np.array_equal(p["mu"], golden[f"fp{i}_mu"]), i


def test_chebav_restatement_bitwise(golden):
    ia, ja, a = O.lap_csr(20, 20, 1)
    pol = O.find_pol([0.6, 1.2, 0.0, 8.0])
    y = O.cheb_av(pol, ia, ja, a, golden["chebav_v"])
    assert np.array_equal(y, golden["chebav_y"])


def test_kpmdos_restatement(golden):
    ia, ja, a = O.lap_csr(20, 20, 1)
    probes = O.seeded_rademacher(6, 400, 7)
    mu, ec = O.kpmdos(40, 1, probes, [0.6, 1.2, 0.0, 8.0], ia, ja, a)
    ref = golden["kpm20_mu"]
    assert np.max(np.abs(mu - ref)) <= 1e-13 * np.max(np.abs(ref))
    assert abs(ec - golden["kpm20_ecnt"][0]) <= 1e-12 * abs(golden["kpm20_ecnt"][0])
    ia, ja, a = O.lap_csr(8, 8, 8)
    probes = O.seeded_rademacher(5, 512, 9)
    mu, ec = O.kpmdos(60, 1, probes, [0.6, 2.0, 0.0, 12.0], ia, ja, a)
    ref = golden["kpm8_mu"]
    assert np.max(np.abs(mu - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_spslicer_restatement_bitwise(golden):
    for key, mukey, ekey, iv, nint in (("sli20", "kpm20_mu", "kpm20_ecnt", [0.6, 1.2, 0.0, 8.0], 4),
                                       ("sli8", "kpm8_mu", "kpm8_ecnt", [0.6, 2.0, 0.0, 12.0], 5)):
        err, sli = O.spslicer(golden[mukey], iv, nint, int(10 * golden[ekey][0]))
        assert err == 0
        assert np.array_equal(sli, golden[key]), key


def test_cheblan_nr_restatement(golden):
    ia, ja, a = O.lap_csr(20, 20, 1)
    pol = O.find_pol([0.6, 1.2, 0.0, 8.0])
    lam, Y, res, _ = O.cheblan_nr([0.6, 1.2, 0.0, 8.0], 400, 1e-8, golden["chebav_v"], pol, ia, ja, a)
    assert len(lam) == len(golden["nr20_lam"]) == len(O.exeiglap3(20, 20, 1, 0.6, 1.2))
    assert np.max(np.abs(np.sort(lam) - golden["nr20_lam"])) < 1e-12
    assert np.all(res < 1e-8)


BOUND_CASES = {
    "lap2d": lambda: O.lap_csr(30, 30, 1),
    "lap3d": lambda: O.lap_csr(12, 11, 10),
    "rspd": lambda: __import__("evsl_b200.workloads", fromlist=["x"]).random_spd_csr(3000, 16, 5),
}


@pytest.mark.parametrize("name", sorted(BOUND_CASES))
def test_lan_bounds_restatement(golden, name):
    ia, ja, a = BOUND_CASES[name]()
    lo, hi = O.lan_bounds(40, O.seeded_normal(len(ia) - 1, 77), ia, ja, a)
    ref = golden[f"lb_{name}"]
    scale = abs(ref[0]) + abs(ref[1])
    assert abs(lo - ref[0]) <= 1e-12 * scale and abs(hi - ref[1]) <= 1e-12 * scale


def test_cheb_si_restatement(golden):
    cfg = golden["si1_cfg"]
    iv, nev, seed = list(cfg[:4]), int(cfg[4]), int(cfg[5])
    ia, ja, a = O.lap_csr(41, 53, 1)
    n = len(ia) - 1
    pol = O.find_pol(iv, damping=0, thresh_int=0.5)
    lam, Y, res = O.cheb_si(nev, iv, 1000, 1e-8, O.seeded_normal(n * nev, seed).reshape(nev, n), pol, ia, ja, a)
    assert len(lam) == len(golden["si1_lam"]) == len(O.exeiglap3(41, 53, 1, iv[0], iv[1]))
    assert np.max(np.abs(np.sort(lam) - golden["si1_lam"])) < 1e-12
    assert np.all(res < 1e-8)


def test_random_spd_matrix():
    from evsl_b200 import workloads as W

    ia, ja, a = W.random_spd_csr(400, 8, 3)
    n = len(ia) - 1
    M = np.zeros((n, n))
    for i in range(n):
        cols = ja[ia[i]:ia[i + 1]]
        assert np.all(np.diff(cols) > 0)
        M[i, cols] = a[ia[i]:ia[i + 1]]
    assert np.array_equal(M, M.T)
    ev = np.linalg.eigvalsh(M)
    lo, hi = W.gershgorin_bounds(ia, ja, a)
    assert ev[0] > 0 and lo <= ev[0] and hi >= ev[-1]


def test_exact_spectrum_counts(golden):
    ex = O.exeiglap3(100, 100, 1, 0.6, 0.9)
    assert len(ex) == 260 == len(golden["cfg1_lam"])
    assert np.max(np.abs(ex - golden["cfg1_lam"])) < 1e-13


def test_lap_csr_structure():
    ia, ja, a = O.lap_csr(4, 3, 2)
    n = 24
    assert len(ia) == n + 1 and ia[-1] == len(ja)
    dense = np.zeros((n, n))
    for r in range(n):
        for j in range(ia[r], ia[r + 1]):
            dense[r, ja[j]] = a[j]
        assert np.all(np.diff(ja[ia[r]:ia[r + 1]]) > 0)
    assert np.allclose(dense, dense.T)
    ev = np.linalg.eigvalsh(dense)
    assert np.allclose(ev, O.exeiglap3(4, 3, 2, -1, 100), atol=1e-12)


@pytest.mark.skipif(not HAVE_REF, reason="reference build oracle/_ref not present")
def test_reference_library_matches_restatement():
    R = O.RefLib()
    ia, ja, a = R.lap_csr(12, 9, 3)
    ia2, ja2, a2 = O.lap_csr(12, 9, 3)
    assert np.array_equal(ia, ia2) and np.array_equal(ja, ja2) and np.array_equal(a, a2)
    R.set_csr(ia, ja, a)
    x = np.random.default_rng(3).standard_normal(len(ia) - 1)
    assert np.array_equal(R.matvec(x), O.csr_matvec(ia, ja, a, x))
    iv = [0.9, 2.2, 0.0, 12.0]
    rc, pol = R.find_pol(iv)
    y = R.chebav(pol, x)
    assert np.array_equal(y, O.cheb_av(O.find_pol(iv), ia, ja, a, x))
    R.free_pol(pol)


@pytest.mark.parametrize("dims, M", [((12, 10, 9), 60), ((40, 40, 1), 31)])
def test_kpm_product_identities_restatement(dims, M):
    """The product-identity form of the KPM moments (two per matrix product)
    equals the direct per-degree dots to rounding, odd and even counts."""
    ia, ja, a = O.lap_csr(*dims)
    n = len(ia) - 1
    probes = O.seeded_normal(n * 4, 5).reshape(4, n)
    iv = [0.6, 1.2, 0.0, 12.0 if dims[2] > 1 else 8.0]
    d0 = O.kpm_raw_dots(M, probes, iv, ia, ja, a)
    d1 = O.kpm_raw_dots_identities(M, probes, iv, ia, ja, a)
    assert np.max(np.abs(d1 - d0)) <= 1e-12 * np.max(np.abs(d0))


@pytest.mark.skipif(not HAVE_REF, reason="reference build not present")
def test_find_pol_restatement_bitwise_on_random_intervals():
    """The restated filter design equals the reference build's bit for bit
    on seeded random mid-spectrum intervals, all three dampings, designed
    and forced degrees: its sines, cosines and sums are taken in the
    reference's scalar order (C library trigonometry, left-to-right sums)."""
    R = O.RefLib()
    rng = np.random.default_rng(17)
    for i in range(40):
        x = np.sort(rng.uniform(0.05, 0.95, 2))
        lo, hi = -3.0 + rng.uniform(), 9.0 + rng.uniform()
        iv = [lo + x[0] * (hi - lo), lo + x[1] * (hi - lo), lo, hi]
        # a forced degree at or above the design loop's starting degree 2 + 0.5 / (half-width in [-1, 1])
        dmin = int(2 + 0.5 / ((x[1] - x[0]) * 2.0)) + 1
        kw = dict(damping=int(i % 3), max_deg=400, deg=(0 if i % 2 else int(rng.integers(dmin, dmin + 120))))
        rc, pol = R.find_pol(iv, **kw)
        ref = R.pol_dict(pol)
        R.free_pol(pol)
        got = O.find_pol(iv, **kw)
        assert rc == 0 and got["deg"] == ref["deg"] and got["type"] == ref["type"], (i, iv, kw)
        assert np.array_equal(got["mu"], ref["mu"]), (i, iv, kw)
        assert got["gam"] == ref["gam"] and got["bar"] == ref["bar"], (i, iv, kw)
