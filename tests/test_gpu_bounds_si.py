"""GPU parity tests for the spectrum-bound estimators (LanBounds,
LanTrbounds), the block filter and filtered subspace iteration (ChebSI),
through the C ABI, against golden fixtures from the reference build.

Tolerances (written per test):
  * block filter: every column bitwise equal to single-vector ChebAv;
  * LanBounds: |bound - bound_ref| <= 1e-9 (|lo_ref| + |hi_ref|) (only the
    summation order of the dot products differs; the Lanczos vectors lose
    orthogonality at the same rate);
  * LanTrbounds: |bound - bound_ref| <= 1e-7 (|lo_ref| + |hi_ref|) (the
    restarted run converges to tol 1e-8 relative), and the bounds contain
    the exact spectrum;
  * ChebSI: eigenvalue count exact against the reference and the analytic
    spectrum, eigenvalues within 1e-10 x (spectral width), residuals < tol.
"""
import numpy as np
import pytest

from evsl_b200 import workloads as W
from oracle import evsl_oracle as O

pytestmark = pytest.mark.gpu

BOUND_CASES = {
    "lap2d": lambda: O.lap_csr(30, 30, 1),
    "lap3d": lambda: O.lap_csr(12, 11, 10),
    "rspd": lambda: W.random_spd_csr(3000, 16, 5),
}


def _spectrum(ia, ja, a):
    n = len(ia) - 1
    M = np.zeros((n, n))
    for i in range(n):
        M[i, ja[ia[i]:ia[i + 1]]] = a[ia[i]:ia[i + 1]]
    return np.linalg.eigvalsh(M)


@pytest.mark.parametrize("name", sorted(BOUND_CASES))
def test_lan_bounds_match_reference(gpu_lib, golden, name):
    ia, ja, a = BOUND_CASES[name]()
    gpu_lib.set_csr(ia, ja, a)
    v = O.seeded_normal(len(ia) - 1, 77)
    lo, hi = gpu_lib.lan_bounds(40, v)
    ref = golden[f"lb_{name}"]
    scale = abs(ref[0]) + abs(ref[1])
    assert abs(lo - ref[0]) <= 1e-9 * scale and abs(hi - ref[1]) <= 1e-9 * scale


@pytest.mark.parametrize("bndtype", [1, 2])
@pytest.mark.parametrize("name", sorted(BOUND_CASES))
def test_lan_trbounds_match_reference(gpu_lib, golden, name, bndtype):
    ia, ja, a = BOUND_CASES[name]()
    gpu_lib.set_csr(ia, ja, a)
    v = O.seeded_normal(len(ia) - 1, 77)
    lo, hi = gpu_lib.lan_trbounds(30, 200, 1e-8, v, bndtype)
    ref = golden[f"ltb{bndtype}_{name}"]
    scale = abs(ref[0]) + abs(ref[1])
    assert abs(lo - ref[0]) <= 1e-7 * scale and abs(hi - ref[1]) <= 1e-7 * scale
    ev = _spectrum(ia, ja, a)
    assert lo <= ev[0] + 1e-8 * scale and hi >= ev[-1] - 1e-8 * scale


def test_block_filter_is_columnwise_chebav(gpu_lib):
    for dims in ((41, 53, 1), (13, 12, 11)):
        ia, ja, a = O.lap_csr(*dims)
        gpu_lib.set_csr(ia, ja, a)
        n = len(ia) - 1
        iv = [0.4, 0.5, 0.0, 8.0 if dims[2] == 1 else 12.0]
        pol = gpu_lib.find_pol(iv, damping=0, thresh_int=0.5)
        for ncols in (1, 5, 8, 19):
            V = O.seeded_normal(n * ncols, 3 + ncols).reshape(ncols, n)
            Y = gpu_lib.chebav_block(pol, V)
            for c in range(ncols):
                assert np.array_equal(Y[c], gpu_lib.chebav(pol, V[c]))
        gpu_lib.free_pol(pol)


@pytest.mark.parametrize("case", ["si1", "si2"])
def test_cheb_si_matches_reference(gpu_lib, golden, case):
    """The reference's subspace-iteration test problem: 2-D 41x53 Laplacian,
    damping 0, thresh_int 0.5, tol 1e-8, maxit 1000, seeded start block."""
    cfg = golden[f"{case}_cfg"]
    iv, nev, seed = list(cfg[:4]), int(cfg[4]), int(cfg[5])
    ia, ja, a = O.lap_csr(41, 53, 1)
    gpu_lib.set_csr(ia, ja, a)
    n = len(ia) - 1
    pol = gpu_lib.find_pol(iv, damping=0, thresh_int=0.5)
    V0 = O.seeded_normal(n * nev, seed).reshape(nev, n)
    lam, Y, res = gpu_lib.cheb_si(nev, iv, 1000, 1e-8, V0, pol)
    ref = golden[f"{case}_lam"]
    exact = O.exeiglap3(41, 53, 1, iv[0], iv[1])
    assert len(lam) == len(ref) == len(exact)
    lam = np.sort(lam)
    assert np.max(np.abs(lam - ref)) <= 1e-10 * 8.0
    assert np.max(np.abs(lam - exact)) <= 1e-10 * 8.0
    assert np.all(res < 1e-8)
    G = Y @ Y.T
    assert np.max(np.abs(G - np.eye(len(lam)))) < 1e-8
    for i in range(len(lam)):
        r = O.csr_matvec(ia, ja, a, Y[i]) - (Y[i] @ O.csr_matvec(ia, ja, a, Y[i])) * Y[i]
        assert np.linalg.norm(r) < 1e-8
    gpu_lib.free_pol(pol)


def test_cheb_si_edge_cases(gpu_lib):
    ia, ja, a = O.lap_csr(20, 20, 1)
    gpu_lib.set_csr(ia, ja, a)
    pol = gpu_lib.find_pol([0.6, 1.2, 0.0, 8.0])
    V0 = O.seeded_normal(400 * 4, 2).reshape(4, 400)
    # interval outside [lmin, lmax]: nothing found, return code 0
    lam, Y, res = gpu_lib.cheb_si(4, [9.0, 10.0, 0.0, 8.0], 50, 1e-8, V0, pol)
    assert len(lam) == 0
    gpu_lib.free_pol(pol)


@pytest.mark.parametrize("mode", ["persistent", "wave"])
def test_bounded_waits_time_out_and_library_recovers(gpu_lib, mode):
    """Failure path of the device-side waits: with a wait limit of one poll,
    the grid barriers of the single-launch filter (or the dependency waits of
    the pipelined filter) give up; the call returns EVSLX_ERR_TIMEOUT (-105),
    every block leaves, and afterwards -- default limits restored -- the
    same filter gives the reference's vector bit for bit."""
    import evsl_b200 as E

    ia, ja, a = O.lap_csr(60, 50, 40)
    n = len(ia) - 1
    iv = [0.6, 1.2, 0.0, 12.0]
    v = O.seeded_normal(n, 3)
    y_ref = O.cheb_av(O.find_pol(iv, deg=40), ia, ja, a, v)
    gpu_lib.set_csr(ia, ja, a)
    pol = gpu_lib.find_pol(iv, deg=40)
    on = (gpu_lib.set_filter_persistent if mode == "persistent" else gpu_lib.set_filter_wave)
    try:
        on(True)
        gpu_lib.set_wait_limit(1)
        codes = []
        for _ in range(3):
            try:
                gpu_lib.chebav(pol, v)
                codes.append(0)
            except E.EvslError as e:
                codes.append(-105 if "returned -105" in str(e) else str(e))
                assert "within its bound" in gpu_lib.last_error()
        assert -105 in codes, codes
        assert all(c in (0, -105) for c in codes), codes
        gpu_lib.set_wait_limit(0)
        assert np.array_equal(gpu_lib.chebav(pol, v), y_ref)
        on(False)
        assert np.array_equal(gpu_lib.chebav(pol, v), y_ref)
    finally:
        gpu_lib.set_wait_limit(0)
        on(False)
        gpu_lib.free_pol(pol)
