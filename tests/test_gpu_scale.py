"""Parity at the benchmark configurations' sizes, against reference results
computed by the reference build (tests/golden/make_golden.py scale).

* kpmdos with the drop-in slicing configuration's settings: the 3-D
  Laplacian 100^3 (n = 10^6), 300 moments, Jackson damping, 30 seeded
  Rademacher probes (SRC/spslice.c:29-148).  The library takes two moments
  per block product from the Chebyshev product identities
  (mu_2k = 2<w_k, w_k> - mu_0, mu_2k+1 = 2<w_k+1, w_k> - mu_1); the
  reference forms one dot per degree.
* kpmdos on the 2-million-row random sparse SPD matrix of the
  mixed-precision configuration, 100 moments, 8 seeded Gaussian probes.

Bars: ||mu - mu_ref||_inf <= 1e-12 ||mu_ref||_inf (normwise), and per moment
|mu_k - mu_ref,k| <= 1e-12 |mu_ref,k| for every moment above the round-off
level of the dot products, |mu_ref,k| >= 1e-3 ||mu_ref||_inf (below it the
reference's own sequential dots carry errors of that relative size);
ecnt 1e-10 relative.  Both errors are printed.

For the Rademacher probes on 10^6 rows the reference's own moments are off
by ~1.5e-12 of max |mu|: every probe entry has the same magnitude, so the
rounding of its sequential FP64 dot over 10^6 terms is systematic.  That
case is therefore checked against the moments of the reference's own FP64
recurrence with every dot accumulated in extended precision (the
`exactdot` fixture): the library must be within the bars of those, and its
distance to the reference's printed moments must not exceed the reference's
own distance to them by more than 1e-13 of max |mu|.
"""
import os

import numpy as np
import pytest

from evsl_b200 import workloads as W
from oracle import evsl_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "evsl_ref_golden_scale.npz"))


def _moment_errors(mu, ref):
    norm = np.max(np.abs(ref))
    normwise = np.max(np.abs(mu - ref)) / norm
    big = np.abs(ref) >= 1e-3 * norm
    rel = np.abs(mu - ref)[big] / np.abs(ref)[big]
    return normwise, float(np.max(rel)), int(np.count_nonzero(big))


@pytest.mark.parametrize("doubling", [1, 0])
def test_kpm_config2_settings_match_reference(gpu_lib, G, doubling):
    ia, ja, a = O.lap_csr(*[int(d) for d in G["kpm100_dims"]])
    gpu_lib.set_csr(ia, ja, a)
    n = len(ia) - 1
    probes = O.seeded_rademacher(int(G["kpm100_nvec"]), n, int(G["kpm100_seed"]))
    gpu_lib.lib.evslcu_set_kpm_doubling(doubling)
    try:
        mu, ec = gpu_lib.kpmdos_probes(int(G["kpm100_M"]), 1, probes, list(G["kpm100_intv"]))
    finally:
        gpu_lib.lib.evslcu_set_kpm_doubling(1)
    ref, exact = G["kpm100_mu"], G["kpm100_mu_exactdot"]
    normwise, rel, nbig = _moment_errors(mu, exact)
    ref_norm, ref_rel, _ = _moment_errors(ref, exact)
    print(f"kpm 100^3 ({'product identities' if doubling else 'direct dots'}) vs exact-dot moments: normwise "
          f"{normwise:.2e}, per-moment relative {rel:.2e} over {nbig} of {len(ref)} moments; the reference "
          f"itself: {ref_norm:.2e} / {ref_rel:.2e}; library vs reference {_moment_errors(mu, ref)[0]:.2e}")
    assert normwise <= 1e-12
    assert rel <= 1e-12
    scale = np.max(np.abs(exact))
    assert np.max(np.abs(mu - ref)) <= np.max(np.abs(ref - exact)) + 1e-13 * scale
    assert abs(ec - G["kpm100_ecnt_exactdot"][0]) <= 1e-10 * abs(G["kpm100_ecnt_exactdot"][0])
    assert abs(ec - G["kpm100_ecnt"][0]) <= 1e-10 * abs(G["kpm100_ecnt"][0])


def test_kpm_random_spd_two_million_rows_matches_reference(gpu_lib, G):
    n = int(G["rspd2m_n"])
    ia, ja, a = W.random_spd_csr(n, 16, int(G["rspd2m_seed"]))
    gpu_lib.set_csr(ia, ja, a)
    del ja, a
    nvec = int(G["rspd2m_nvec"])
    probes = O.seeded_normal(n * nvec, int(G["rspd2m_pseed"])).reshape(nvec, n)
    mu, ec = gpu_lib.kpmdos_probes(int(G["rspd2m_M"]), 1, probes, list(G["rspd2m_intv"]))
    ref = G["rspd2m_mu"]
    normwise, rel, nbig = _moment_errors(mu, ref)
    print(f"kpm random SPD n={n}: normwise {normwise:.2e}, per-moment relative {rel:.2e} over {nbig} moments")
    assert normwise <= 1e-12
    assert rel <= 1e-12
    assert abs(ec - G["rspd2m_ecnt"][0]) <= 1e-10 * abs(G["rspd2m_ecnt"][0])
