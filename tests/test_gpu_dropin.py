"""Drop-in check: the reference's own spectrum-slicing driver
(TESTS/PLanN/LapPLanN.c with TESTS/COMMON/{lapl,io,mmio}.c), compiled
unchanged with -DEVSL_USING_CUDA_GPU against this repository's
include/evsl.h and linked to libevsl_b200.so instead of the reference library
(oracle/Makefile builds it as oracle/_ref/LapPLanN_b200.ex where the
reference sources exist; the binary travels with the built library).

The driver runs the whole path through the reference API -- EVSLStart,
evsl_create_csr_gpu, SetAMatrix_device_csr, kpmdos (60 probes, 300 moments),
spslicer, rand_double_device, then per slice set_pol_def / find_pol /
ChebLanNr / sort_double / StatsPrint -- and compares each slice with the
analytic Laplacian spectrum itself.  The test checks its printed counts
(found == exact for every slice) and, from its output file, the eigenvalue
errors against the analytic values (<= 1e-10 x spectral width) and the
residuals (<= the driver's tol, 1e-6).
"""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "LapPLanN_b200.ex")


@pytest.mark.parametrize("args, nslices, width", [
    (["-nx", "16", "-ny", "16", "-nz", "20"], 4, 12.0),                         # the driver's defaults
    (["-nx", "30", "-ny", "30", "-nz", "1", "-a", "0.6", "-b", "1.2", "-nslices", "3"], 3, 8.0),
])
def test_reference_driver_runs_unchanged_on_this_library(tmp_path, args, nslices, width):
    assert os.path.exists(DRIVER), f"{DRIVER} is missing: build it with `make -C oracle` (needs the reference sources)"
    p = subprocess.run([DRIVER] + args, cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    counts = re.findall(r"number of eigenvalues: (\d+), found: (\d+)", p.stdout)
    assert len(counts) == nslices, p.stdout
    assert all(int(a) == int(b) and int(a) > 0 for a, b in counts), counts
    out = open(os.path.join(tmp_path, "OUT", "LapPLanN.out")).read()
    rows = [ln.split() for ln in out.splitlines()]
    rows = [r for r in rows if len(r) == 4 and all(re.fullmatch(r"[-+]?\d\.\d+e[-+]\d+", t) for t in r)]
    assert len(rows) >= sum(min(int(a), 52) for a, _ in counts) - nslices
    assert max(abs(float(r[3])) for r in rows) <= 1e-10 * width
    assert max(float(r[1]) for r in rows) <= 1e-6


REF_CUDA_DRIVER = os.path.join(ROOT, "oracle", "_ref", "cuda", "LapPLanN_refcuda.ex")


def test_reference_cuda_build_under_the_same_driver(tmp_path):
    """The same driver on the reference's own CUDA build (cuSPARSE / cuBLAS,
    `make -C oracle cuda`) and on this library, on one problem: both find
    every eigenvalue of every slice (counts from the driver's own check
    against the analytic spectrum), and this library's run reports the
    filter and reorthogonalisation times the reference's StatsPrint
    reports."""
    if not os.path.exists(REF_CUDA_DRIVER):
        pytest.skip("the reference CUDA build is not built (make -C oracle cuda)")
    args = ["-nx", "30", "-ny", "30", "-nz", "30", "-a", "0.5", "-b", "0.9", "-nslices", "2"]
    found = {}
    for name, exe in (("ref", REF_CUDA_DRIVER), ("b200", DRIVER)):
        d = tmp_path / name
        d.mkdir()
        p = subprocess.run([exe] + args, cwd=d, capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stdout + p.stderr
        counts = re.findall(r"number of eigenvalues: (\d+), found: (\d+)", p.stdout)
        assert len(counts) == 2 and all(int(a) == int(b) > 0 for a, b in counts), (name, counts)
        found[name] = sum(int(a) for a, _ in counts)
        out = open(os.path.join(d, "OUT", "LapPLanN.out")).read()
        if name == "b200":
            pol = re.findall(r"Pol\(A\)\*v\s+:\s+([0-9.]+)", out)
            reo = re.findall(r"Reorthogonalization\s+:\s+([0-9.]+)", out)
            assert len(pol) == 2 and all(float(t) > 0 for t in pol), out[-800:]
            assert len(reo) == 2 and all(float(t) > 0 for t in reo), out[-800:]
    # the slices come from each library's own random probes, so their end
    # points differ; the eigenvalues of [a, b] are the same set
    assert found["ref"] == found["b200"]
