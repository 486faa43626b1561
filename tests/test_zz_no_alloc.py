"""The allocation-free KPM entry point, evslx_kpmdos_probes_noalloc.

Who needs it: a process that reserves the GPU's memory up front -- resident
matrices and Lanczos bases under a fixed HBM budget -- must not call
cudaMalloc/cudaFree while it serves a density-of-states request; that would
break the budget and synchronise the device in the middle of other requests.
This entry point keeps all its device scratch in one fixed 32 MiB array
inside the library and allocates nothing per call.

The test calls it through the C ABI twice in a row and checks both results
against the allocating entry point (evslx_kpmdos_probes) with the KPM
tolerance used everywhere in these tests (moments normwise 1e-12 relative,
count 1e-10 relative).  It lives in its own file, collected last, so that a
run stopping at the first failure has already run every other test; it also
passes when run alone in a fresh process (the first call then performs the
one-time address lookup).
"""
import ctypes as C

import numpy as np
import pytest

import evsl_b200
from oracle import evsl_oracle as O

pytestmark = pytest.mark.gpu

_dp = C.POINTER(C.c_double)


def _kpm(lib, fn, Mdeg, damping, nvec, intv, dprobes):
    mu = np.zeros(Mdeg + 1)
    ec = C.c_double()
    iv = np.ascontiguousarray(intv, dtype=np.float64)
    rc = fn(Mdeg, damping, nvec, iv.ctypes.data_as(_dp), dprobes.ptr, mu.ctypes.data_as(_dp), C.byref(ec))
    return rc, mu, ec.value


def _check_twice(gpu_lib, nvec, Mdeg, intv, seed):
    n = gpu_lib.n
    probes = O.seeded_rademacher(nvec, n, seed)
    dprobes = evsl_b200.DeviceBuffer.from_host(gpu_lib.lib, probes)
    rc, mu_ref, ec_ref = _kpm(gpu_lib.lib, gpu_lib.lib.evslx_kpmdos_probes, Mdeg, 1, nvec, intv, dprobes)
    assert rc == 0, gpu_lib.last_error()
    for _ in range(2):
        rc, mu, ec = _kpm(gpu_lib.lib, gpu_lib.lib.evslx_kpmdos_probes_noalloc, Mdeg, 1, nvec, intv, dprobes)
        assert rc == 0, gpu_lib.last_error()
        assert np.max(np.abs(mu - mu_ref)) <= 1e-12 * np.max(np.abs(mu_ref))
        assert abs(ec - ec_ref) <= 1e-10 * abs(ec_ref)


@pytest.mark.parametrize("nvec", [24, 64, 100, 128])
def test_noalloc_kpm_matches_allocating_entry_point(gpu_lib, nvec):
    """Up to 32, 64 and 128 probes per launch (the three kernel forms)."""
    ia, ja, a = O.lap_csr(30, 30, 4)
    gpu_lib.set_csr(ia, ja, a)
    _check_twice(gpu_lib, nvec, 120, [0.8, 2.5, 0.0, 12.0], 13)


def test_noalloc_kpm_just_under_its_scratch(gpu_lib):
    """The largest 2-D grid whose scratch need fits the fixed array at 128
    probes: it runs and matches; one row more per column is rejected."""
    need = gpu_lib.lib.evslcu_kpm_noalloc_need
    need.argtypes = [C.c_int, C.c_int, C.c_int]
    need.restype = C.c_size_t
    cap_fn = gpu_lib.lib.evslcu_kpm_noalloc_capacity
    cap_fn.restype = C.c_size_t
    cap = cap_fn()
    nx, Mdeg, nvec = 100, 60, 128
    ny = max(k for k in range(1, 200) if need(nx * k, Mdeg, nvec) <= cap)
    assert need(nx * ny, Mdeg, nvec) > 0.98 * cap and need(nx * (ny + 1), Mdeg, nvec) > cap
    ia, ja, a = O.lap_csr(nx, ny, 1)
    gpu_lib.set_csr(ia, ja, a)
    _check_twice(gpu_lib, nvec, Mdeg, [0.8, 2.5, 0.0, 8.0], 14)
    ia, ja, a = O.lap_csr(nx, ny + 1, 1)
    gpu_lib.set_csr(ia, ja, a)
    dprobes = evsl_b200.DeviceBuffer(gpu_lib.lib, 8 * nx * (ny + 1) * nvec)
    rc, mu, ec = _kpm(gpu_lib.lib, gpu_lib.lib.evslx_kpmdos_probes_noalloc, Mdeg, 1, nvec, [0.8, 2.5, 0.0, 8.0],
                      dprobes)
    assert rc != 0 and "scratch" in gpu_lib.last_error()


def test_noalloc_kpm_rejects_sizes_beyond_its_scratch(gpu_lib):
    ia, ja, a = O.lap_csr(450, 450, 1)
    gpu_lib.set_csr(ia, ja, a)
    n = len(ia) - 1
    dprobes = evsl_b200.DeviceBuffer(gpu_lib.lib, 8 * n * 30)
    rc, mu, ec = _kpm(gpu_lib.lib, gpu_lib.lib.evslx_kpmdos_probes_noalloc, 50, 1, 30, [0.5, 1.0, 0.0, 8.0], dprobes)
    assert rc != 0
    assert "scratch" in gpu_lib.last_error()
