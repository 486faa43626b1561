"""Generate the golden fixtures in tests/golden/ from the reference EVSL CPU
library (oracle/_ref/libevsl_ref.so, built by `make -C oracle` from the
reference sources).  Run from the repository root:

    python tests/golden/make_golden.py          # evsl_ref_golden.npz
    python tests/golden/make_golden.py scale    # evsl_ref_golden_scale.npz
    python tests/golden/make_golden.py scale-exact   # (re)adds its exact-dot KPM moments

Every input is seeded; probe and start vectors are injected into the
reference through its rand_double_device hook (oracle/ref_hooks.c).  The
`scale` fixtures hold reference results at the benchmark configurations'
sizes (minutes of reference CPU time): kpmdos on the 3-D Laplacian 100^3 with
300 moments and 30 probes, and on the 2-million-row random SPD matrix with 100
moments and 8 Gaussian probes; ChebLanNr on a 20,000-row matrix from the
same random SPD generator with its exact eigenvalues from a dense solve.
"""
import gzip
import os
import shutil
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import evsl_oracle as O  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden")
MM_DIR = os.path.join(OUT, "mm")
REF_ROOT = os.environ.get("EVSL_REFERENCE", "/root/reference/EVSL_1.1.1")
REF_MATRICES = os.path.join(REF_ROOT, "MATRICES")

# Scale fixtures: (name, value) of the seeds and sizes the GPU tests repeat.
SCALE = {
    "kpm100_dims": (100, 100, 100), "kpm100_M": 300, "kpm100_nvec": 30, "kpm100_seed": 41,
    "kpm100_intv": (0.6, 1.2, 0.0, 12.0),
    "rspd_n": 20000, "rspd_seed": 33, "rspd_vseed": 34, "rspd_lo_index": 1000, "rspd_count": 50,
    "rspd2m_n": 2000000, "rspd2m_seed": 3, "rspd2m_M": 100, "rspd2m_nvec": 8, "rspd2m_pseed": 45,
}


def _fmt(v, rng):
    """Value text in a few of the notations Matrix-Market files use."""
    k = rng.integers(0, 3)
    if k == 0:
        return repr(float(v))
    if k == 1:
        return "%.6e" % v
    return "%.4f" % v


def write_mm_fixtures():
    """Small Matrix-Market files covering the reader's cases (seeded)."""
    os.makedirs(MM_DIR, exist_ok=True)
    rng = np.random.default_rng(31)
    files = {}
    # general real with comments, unsorted entries and duplicated positions
    n, m = 40, 200
    r = rng.integers(1, n + 1, m)
    c = rng.integers(1, n + 1, m)
    r[-10:], c[-10:] = r[:10], c[:10]
    lines = ["%%MatrixMarket matrix coordinate real general", "% seeded test matrix", "%", f"{n} {n} {m}"]
    lines += [f"{r[k]} {c[k]} {_fmt(rng.standard_normal(), rng)}" for k in range(m)]
    files["gen_dup"] = lines
    # symmetric real: lower triangle with the diagonal, random order
    n = 50
    pos = [(i, j) for i in range(1, n + 1) for j in range(1, i + 1) if i == j or rng.random() < 0.08]
    rng.shuffle(pos)
    lines = ["%%MatrixMarket matrix coordinate real symmetric", f"{n} {n} {len(pos)}"]
    lines += [f"{i} {j} {_fmt(rng.uniform(-1, 1) + (4.0 if i == j else 0.0), rng)}" for i, j in pos]
    files["sym"] = lines
    # integer general with an upper-case banner
    n, m = 30, 90
    lines = ["%%MatrixMarket MATRIX Coordinate INTEGER General", f"{n} {n} {m}"]
    lines += [f"{rng.integers(1, n + 1)} {rng.integers(1, n + 1)} {rng.integers(-9, 10)}" for _ in range(m)]
    files["int_upper"] = lines
    # skew-symmetric: read as stored (not expanded)
    n = 20
    pos = [(i, j) for i in range(2, n + 1) for j in range(1, i) if rng.random() < 0.2]
    lines = ["%%MatrixMarket matrix coordinate real skew-symmetric", f"{n} {n} {len(pos)}"]
    lines += [f"{i} {j} {_fmt(rng.standard_normal(), rng)}" for i, j in pos]
    files["skew"] = lines
    # rejected: pattern field, non-square, short file
    files["pattern"] = ["%%MatrixMarket matrix coordinate pattern general", "3 3 2", "1 1", "2 3"]
    files["rect"] = ["%%MatrixMarket matrix coordinate real general", "5 6 2", "1 1 1.0", "2 3 2.0"]
    files["short"] = ["%%MatrixMarket matrix coordinate real general", "4 4 10"] + [f"{k} {k} 1.5" for k in
                                                                                       range(1, 5)]
    for name, lines in files.items():
        with open(os.path.join(MM_DIR, name + ".mtx"), "w") as f:
            f.write("\n".join(lines) + "\n")
    # the reference's own test matrix (stiffness matrix, n = 5795), compressed
    with open(os.path.join(REF_MATRICES, "A.mtx"), "rb") as src, \
            gzip.GzipFile(os.path.join(MM_DIR, "A.mtx.gz"), "wb", mtime=0) as dst:
        shutil.copyfileobj(src, dst)
    return sorted(files)

FIND_POL_CASES = [
    # (intv, damping, thresh_int, thresh_ext, max_deg)
    ([0.6, 0.9, 0.0, 8.0], 2, 0.8, 0.2, 3000),     # config-1 filter (middle interval)
    ([0.6, 1.2, 0.0, 12.0], 2, 0.8, 0.2, 3000),    # config-2 interval
    ([0.6, 0.69331, 0.0, 12.0], 2, 0.8, 0.2, 3000),
    ([0.6, 0.604, 0.0, 12.0], 2, 0.8, 0.2, 3000),  # narrow, high degree
    ([0.0, 0.3, 0.0, 8.0], 2, 0.8, 0.2, 3000),     # left end interval
    ([7.5, 8.0, 0.0, 8.0], 2, 0.8, 0.2, 3000),     # right end interval
    ([1.0, 2.0, 0.0, 8.0], 1, 0.8, 0.2, 3000),     # Jackson damping
    ([1.0, 2.0, 0.0, 8.0], 0, 0.8, 0.2, 3000),     # no damping
    ([-0.5, 0.3, 0.0, 8.0], 2, 0.8, 0.2, 3000),    # interval adjusted to bounds
]


def main():
    R = O.RefLib()
    out = {}
    # ---- find_pol ------------------------------------------------------------
    for i, (iv, damp, ti, te, md) in enumerate(FIND_POL_CASES):
        rc, pol = R.find_pol(iv, damping=damp, thresh_int=ti, thresh_ext=te, max_deg=md)
        d = R.pol_dict(pol)
        out[f"fp{i}_intv"] = np.array(iv)
        out[f"fp{i}_cfg"] = np.array([damp, ti, te, md], dtype=np.float64)
        out[f"fp{i}_scal"] = np.array([d["type"], d["deg"], d["cc"], d["dd"], d["gam"], d["bar"]])
        out[f"fp{i}_mu"] = d["mu"]
        R.free_pol(pol)
    # ---- ChebAv on a 20x20 Laplacian --------------------------------------------
    ia, ja, a = R.lap_csr(20, 20, 1)
    R.set_csr(ia, ja, a)
    iv = [0.6, 1.2, 0.0, 8.0]
    rc, pol = R.find_pol(iv)
    v = O.seeded_normal(400, 101)
    out["chebav_v"] = v
    out["chebav_y"] = R.chebav(pol, v)
    # ---- ChebLanNr / ChebLanTr on the 20x20 Laplacian ------------------------------
    rc, (lam, W, res) = R.cheblan_nr(iv, 400, 1e-8, v, pol)
    out["nr20_lam"] = np.sort(lam)
    out["nr20_res"] = res
    rc, (lam, W, res) = R.cheblan_tr(100, 30, iv, 300, 1e-8, v, pol)
    out["tr20_lam"] = np.sort(lam)
    out["tr20_res"] = res
    R.free_pol(pol)
    # ---- kpmdos + spslicer on the 20x20 Laplacian and an 8^3 Laplacian ------------
    probes = O.seeded_rademacher(6, 400, 7)
    rc, mu, ec = R.kpmdos(40, 1, probes, [0.6, 1.2, 0.0, 8.0])
    out["kpm20_probes_seed"] = np.array([7, 6])
    out["kpm20_mu"] = mu
    out["kpm20_ecnt"] = np.array([ec])
    rc, sli = R.spslicer(mu, [0.6, 1.2, 0.0, 8.0], 4, int(10 * ec))
    out["sli20"] = sli
    ia, ja, a = R.lap_csr(8, 8, 8)
    R.set_csr(ia, ja, a)
    probes = O.seeded_rademacher(5, 512, 9)
    rc, mu, ec = R.kpmdos(60, 1, probes, [0.6, 2.0, 0.0, 12.0])
    out["kpm8_mu"] = mu
    out["kpm8_ecnt"] = np.array([ec])
    rc, sli = R.spslicer(mu, [0.6, 2.0, 0.0, 12.0], 5, int(10 * ec))
    out["sli8"] = sli
    # ---- config 1: 2-D 100x100 Laplacian, [0.6, 0.9], ChebLanNr -------------------
    ia, ja, a = R.lap_csr(100, 100, 1)
    R.set_csr(ia, ja, a)
    iv = [0.6, 0.9, 0.0, 8.0]
    rc, pol = R.find_pol(iv, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=3000)
    v = O.seeded_normal(10000, 1234)
    rc, (lam, W, res) = R.cheblan_nr(iv, 2000, 1e-8, v, pol)
    out["cfg1_lam"] = np.sort(lam)
    out["cfg1_res_max"] = np.array([res.max()])
    out["cfg1_vinit_seed"] = np.array([1234])
    R.free_pol(pol)
    # ---- spectrum bounds: LanBounds / LanTrbounds (simple and Kato-Temple) ----
    from evsl_b200 import workloads as W

    cases = [("lap2d", R.lap_csr(30, 30, 1)), ("lap3d", R.lap_csr(12, 11, 10)),
             ("rspd", W.random_spd_csr(3000, 16, 5))]
    for name, (ia, ja, a) in cases:
        R.set_csr(ia, ja, a)
        v = O.seeded_normal(len(ia) - 1, 77)
        rc, lo, hi = R.lan_bounds(40, v)
        out[f"lb_{name}"] = np.array([lo, hi])
        for bt in (1, 2):
            rc, lo, hi = R.lan_trbounds(30, 200, 1e-8, v, bt)
            out[f"ltb{bt}_{name}"] = np.array([lo, hi])
    # ---- ChebSI on the 41x53 Laplacian of the reference's subspace-iteration test --
    ia, ja, a = R.lap_csr(41, 53, 1)
    R.set_csr(ia, ja, a)
    n = len(ia) - 1
    for name, iv, nev in (("si1", [0.4, 0.5, 0.0, 8.0], 25), ("si2", [0.4, 0.8, 0.0, 8.0], 88)):
        rc, pol = R.find_pol(iv, damping=0, thresh_int=0.5)
        V0 = O.seeded_normal(n * nev, 55).reshape(nev, n)
        rc, (lam, Y, res) = R.cheb_si(nev, iv, 1000, 1e-8, V0, pol)
        out[f"{name}_cfg"] = np.array(iv + [nev, 55])
        out[f"{name}_lam"] = np.sort(lam)
        out[f"{name}_res_max"] = np.array([res.max()])
        R.free_pol(pol)
    # ---- Matrix-Market input: reference read_coo_MM + cooMat_to_csrMat ---------
    for name in write_mm_fixtures():
        rc, n, ir, jc, vv = R.read_coo_mm(os.path.join(MM_DIR, name + ".mtx"), 1, 0)
        out[f"mm_{name}_rc"] = np.array([rc])
        if rc == 0:
            out[f"mm_{name}_coo"] = np.stack([ir, jc]).astype(np.int32)
            out[f"mm_{name}_vv"] = vv
            ia, ja, a = R.coo_to_csr(n, ir, jc, vv, 0)
            out[f"mm_{name}_ia"], out[f"mm_{name}_ja"], out[f"mm_{name}_a"] = ia, ja, a
    # ---- Lanczos DOS + spslicer2 on a 30x30 Laplacian; exDOS ------------------------
    ia, ja, a = R.lap_csr(30, 30, 1)
    R.set_csr(ia, ja, a)
    R.set_seed(11)
    rc, x, y, ec = R.lan_dos(10, 40, 200, [0.5, 2.0, 0.0, 8.0])
    out["ld30_x"], out["ld30_y"], out["ld30_ecnt"] = x, y, np.array([ec])
    out["ld30_sli"] = R.spslicer2(x, y, 4)
    rc, x, y = R.exdos(O.exeiglap3(30, 30, 1, 0.0, 8.0), 300, [0.5, 2.0, 0.0, 8.0])
    out["exdos30_y"] = y
    # ---- the reference's Matrix-Market pipeline on A.mtx (TESTS/PLanN/MMPLanN.c):
    #      LanTrbounds -> LanDos -> spslicer2 -> ChebLanNr per slice, tol 1e-6 --------
    rc, n, ir, jc, vv = R.read_coo_mm(os.path.join(REF_MATRICES, "A.mtx"), 1, 0)
    ia, ja, a = R.coo_to_csr(n, ir, jc, vv, 0)
    R.set_csr(ia, ja, a)
    vinit = O.library_uniform(2024, 0, n)
    rc, lo, hi = R.lan_trbounds(50, 200, 1e-8, vinit, 1)
    R.set_seed(77)
    rc, x, y, ec = R.lan_dos(30, 80, 500, [0.1, 0.3, lo, hi])
    sli = R.spslicer2(x, y, 5)
    out["mmA_bounds"], out["mmA_ecnt"], out["mmA_sli"] = np.array([lo, hi]), np.array([ec]), sli
    counts = []
    lams = []
    for s in range(5):
        nev = int(1 + ec / 5)
        nev = int(1.2 * nev)
        mlan = min(max(5 * nev, 300), n)
        xi = [sli[s], sli[s + 1], lo, hi]
        rc, pol = R.find_pol(xi, damping=2, thresh_int=0.8, thresh_ext=0.2)
        rc, (lam, W, res) = R.cheblan_nr(xi, mlan, 1e-6, vinit, pol)
        counts.append(len(lam))
        lams.append(np.sort(lam))
        R.free_pol(pol)
    out["mmA_counts"] = np.array(counts)
    out["mmA_lam"] = np.concatenate(lams)
    M = np.zeros((n, n))
    for i in range(n):
        M[i, ja[ia[i]:ia[i + 1]]] = a[ia[i]:ia[i + 1]]
    ev = np.linalg.eigvalsh(M)
    out["mmA_exact"] = ev[(ev >= 0.1) & (ev <= 0.3)]
    out["mmA_extremes"] = np.array([ev[0], ev[-1]])
    np.savez_compressed(os.path.join(OUT, "evsl_ref_golden.npz"), **out)
    print("wrote", os.path.join(OUT, "evsl_ref_golden.npz"), "keys:", len(out))


def _exact_dots_worker(args):
    Mdeg, probes, intv, dims = args
    ia, ja, a = O.lap_csr(*dims)
    return O.kpm_raw_dots_exact(Mdeg, probes, intv, ia, ja, a)


def main_scale_exact():
    """Adds to the scale fixtures the KPM moments of the 3-D Laplacian 100^3
    case computed from the reference's own FP64 recurrence with every dot
    product accumulated in extended precision (oracle kpm_raw_dots_exact):
    the reference's moments without the rounding of its sequential FP64 dot
    over 10^6 terms, which for Rademacher probes (equal |v_i|) is systematic
    and reaches ~1.5e-12 of max |mu|."""
    import multiprocessing as mp

    path = os.path.join(OUT, "evsl_ref_golden_scale.npz")
    out = dict(np.load(path))
    S = SCALE
    dims = S["kpm100_dims"]
    n = dims[0] * dims[1] * dims[2]
    probes = O.seeded_rademacher(S["kpm100_nvec"], n, S["kpm100_seed"])
    jobs = [(S["kpm100_M"], probes[m:m + 1], list(S["kpm100_intv"]), dims) for m in range(S["kpm100_nvec"])]
    with mp.get_context("spawn").Pool(6) as pool:
        dots = np.concatenate(pool.map(_exact_dots_worker, jobs), axis=1)
    mu, ec = O.kpm_moments_from_dots(S["kpm100_M"], 1, n, list(S["kpm100_intv"]), dots)
    out["kpm100_mu_exactdot"], out["kpm100_ecnt_exactdot"] = mu, np.array([ec])
    ref = out["kpm100_mu"]
    print("reference vs exact-dot moments: normwise %.2e" % (np.max(np.abs(ref - mu)) / np.max(np.abs(mu))))
    np.savez_compressed(path, **out)
    print("wrote", path, "keys:", len(out))


def main_scale():
    import time

    from evsl_b200 import workloads as W

    R = O.RefLib()
    S = SCALE
    out = {k: np.array(v) for k, v in S.items()}
    # ---- kpmdos at the config-2 settings: 3-D Laplacian 100^3, 300 moments,
    #      Jackson damping, 30 seeded Rademacher probes ------------------------
    t = time.time()
    ia, ja, a = R.lap_csr(*S["kpm100_dims"])
    R.set_csr(ia, ja, a)
    n = len(ia) - 1
    probes = O.seeded_rademacher(S["kpm100_nvec"], n, S["kpm100_seed"])
    rc, mu, ec = R.kpmdos(S["kpm100_M"], 1, probes, list(S["kpm100_intv"]))
    assert rc == 0
    out["kpm100_mu"], out["kpm100_ecnt"] = mu, np.array([ec])
    del probes
    print(f"kpm100: ecnt {ec:.3f} ({time.time() - t:.0f} s)", flush=True)
    # ---- ChebLanNr on a 20,000-row random SPD matrix (the config-3 generator):
    #      50 eigenvalues from the 1000th up, end points at gap midpoints of the
    #      dense spectrum, bounds just outside the extreme eigenvalues ------------
    t = time.time()
    ia, ja, a = W.random_spd_csr(S["rspd_n"], 16, S["rspd_seed"])
    n = len(ia) - 1
    M = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(ia))
    M[rows, ja] = a
    ev = np.linalg.eigvalsh(M)
    del M
    i0, i1 = S["rspd_lo_index"], S["rspd_lo_index"] + S["rspd_count"]
    lo, hi = float(ev[0] - 0.01), float(ev[-1] + 0.01)
    iv = [0.5 * (ev[i0 - 1] + ev[i0]), 0.5 * (ev[i1 - 1] + ev[i1]), lo, hi]
    out["rspd_intv"] = np.array(iv)
    out["rspd_exact"] = ev[i0:i1]
    out["rspd_extremes"] = np.array([ev[0], ev[-1]])
    R.set_csr(ia, ja, a)
    rc, pol = R.find_pol(iv, damping=2, thresh_int=0.8, thresh_ext=0.2)
    v = O.seeded_normal(n, S["rspd_vseed"])
    rc, (lam, Wv, res) = R.cheblan_nr(iv, 3000, 1e-8, v, pol)
    assert rc == 0
    out["rspd_lam"] = np.sort(lam)
    out["rspd_res_max"] = np.array([res.max()])
    out["rspd_deg"] = np.array([R.pol_dict(pol)["deg"]])
    R.free_pol(pol)
    print(f"rspd: {len(lam)} eigenvalues (exact {i1 - i0}), degree {out['rspd_deg'][0]}, "
          f"{time.time() - t:.0f} s", flush=True)
    # ---- kpmdos on the 2-million-row random SPD matrix: 100 moments, Jackson,
    #      8 seeded Gaussian probes, Gershgorin bounds -------------------------------
    t = time.time()
    ia, ja, a = W.random_spd_csr(S["rspd2m_n"], 16, S["rspd2m_seed"])
    n = len(ia) - 1
    glo, ghi = W.gershgorin_bounds(ia, ja, a)
    R.set_csr(ia, ja, a)
    probes = O.seeded_normal(n * S["rspd2m_nvec"], S["rspd2m_pseed"]).reshape(S["rspd2m_nvec"], n)
    iv = [glo + 0.3 * (ghi - glo), glo + 0.35 * (ghi - glo), glo, ghi]
    rc, mu, ec = R.kpmdos(S["rspd2m_M"], 1, probes, iv)
    assert rc == 0
    out["rspd2m_intv"], out["rspd2m_mu"], out["rspd2m_ecnt"] = np.array(iv), mu, np.array([ec])
    print(f"rspd2m: nnz {ia[-1]}, bounds [{glo:.3f}, {ghi:.3f}], ecnt {ec:.1f} ({time.time() - t:.0f} s)",
          flush=True)
    np.savez_compressed(os.path.join(OUT, "evsl_ref_golden_scale.npz"), **out)
    print("wrote", os.path.join(OUT, "evsl_ref_golden_scale.npz"), "keys:", len(out))


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "scale":
        main_scale()
        main_scale_exact()
    elif len(sys.argv) > 1 and sys.argv[1] == "scale-exact":
        main_scale_exact()
    else:
        main()
