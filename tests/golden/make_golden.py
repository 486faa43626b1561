"""Generate the golden fixtures in tests/golden/ from the reference EVSL CPU
library (oracle/_ref/libevsl_ref.so, built by `make -C oracle` from the
reference sources).  Run from the repository root:

    python tests/golden/make_golden.py

Every input is seeded; probe and start vectors are injected into the
reference through its rand_double_device hook (oracle/ref_hooks.c).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import evsl_oracle as O  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden")

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
    np.savez_compressed(os.path.join(OUT, "evsl_ref_golden.npz"), **out)
    print("wrote", os.path.join(OUT, "evsl_ref_golden.npz"), "keys:", len(out))


if __name__ == "__main__":
    main()
