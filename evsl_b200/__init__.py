"""evsl_b200 -- B200-native polynomial-filtered spectrum slicing (EVSL API).

The product is the C-ABI shared library ``libevsl_b200.so`` built from
``evsl_b200/csrc`` (C99 host keeping EVSL's API + CUDA sm_100a kernels).  This
module is a thin ctypes binding of that library, mirroring the reference's
entry points (EVSLStart, SetAMatrix, find_pol, ChebLanNr, ChebLanTr, kpmdos,
spslicer, ChebAv) with numpy arrays for host data.  It contains no numerical
code of its own: every call goes through the library, and importing fails
loudly if the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

__all__ = ["Library", "PolParams", "DeviceBuffer", "EvslError", "library_path", "load", "kpm_accumulate",
           "read_coo_mm", "coo_to_csr_host", "simpson", "spslicer2", "exdos"]

_HERE = os.path.dirname(os.path.abspath(__file__))


def library_path() -> str:
    return os.path.join(_HERE, "libevsl_b200.so")


class EvslError(RuntimeError):
    """A non-zero return code from the library."""


class PolParams(C.Structure):
    """polparams, same layout as the reference (INC/struct.h:68-98)."""

    _fields_ = [
        ("max_deg", C.c_int),
        ("min_deg", C.c_int),
        ("damping", C.c_int),
        ("thresh_ext", C.c_double),
        ("thresh_int", C.c_double),
        ("intvtol", C.c_double),
        ("type", C.c_int),
        ("mu", C.POINTER(C.c_double)),
        ("cc", C.c_double),
        ("dd", C.c_double),
        ("gam", C.c_double),
        ("bar", C.c_double),
        ("deg", C.c_int),
    ]

    def as_dict(self):
        mu = np.ctypeslib.as_array(self.mu, (self.deg + 1,)).copy() if self.mu else None
        return dict(type=self.type, deg=self.deg, cc=self.cc, dd=self.dd, gam=self.gam, bar=self.bar, mu=mu)


class CsrMat(C.Structure):
    """csrMat, same layout as the reference CUDA build (INC/struct.h:29-42)."""

    _fields_ = [
        ("owndata", C.c_int),
        ("nrows", C.c_int),
        ("ncols", C.c_int),
        ("nnz", C.c_int),
        ("ia", C.POINTER(C.c_int)),
        ("ja", C.POINTER(C.c_int)),
        ("a", C.POINTER(C.c_double)),
        ("descr", C.c_void_p),
        ("dBuffer", C.c_char_p),
    ]


class CooMat(C.Structure):
    """cooMat (INC/struct.h:14-21)."""

    _fields_ = [
        ("nrows", C.c_int),
        ("ncols", C.c_int),
        ("nnz", C.c_int),
        ("ir", C.POINTER(C.c_int)),
        ("jc", C.POINTER(C.c_int)),
        ("vv", C.POINTER(C.c_double)),
    ]


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

PREC_FP64 = 0
PREC_MIXED = 1
REQ_SLICE = 1
REQ_KPM = 2


class EvslxResult(C.Structure):
    """evslx_result (include/evslx.h)."""

    _fields_ = [
        ("tag", C.c_uint64),
        ("kind", C.c_int),
        ("rc", C.c_int),
        ("nev", C.c_int),
        ("lam", C.POINTER(C.c_double)),
        ("res", C.POINTER(C.c_double)),
        ("Y", C.c_void_p),
        ("mu", C.POINTER(C.c_double)),
        ("ecnt", C.c_double),
        ("lanczos_steps", C.c_int),
        ("refine_sweeps", C.c_int),
        ("t_submit", C.c_double),
        ("t_start", C.c_double),
        ("t_finish", C.c_double),
    ]


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


_LIB = None


def kpm_accumulate(Mdeg, damping, n, intv, dots):
    """Host-only accumulation of KPM moments from raw dots (Mdeg x nvec);
    needs the library but no GPU."""
    lib = load()
    dots = np.ascontiguousarray(dots, dtype=np.float64)
    mu = np.zeros(Mdeg + 1)
    ec = C.c_double()
    iv = np.ascontiguousarray(intv, dtype=np.float64)
    rc = lib.evslx_kpm_accumulate(Mdeg, damping, dots.shape[1], n, _d(iv), _d(dots), _d(mu), C.byref(ec))
    if rc != 0:
        raise EvslError(f"evslx_kpm_accumulate returned {rc}")
    return mu, ec.value


def read_coo_mm(path, idxin=1, idxout=0):
    """evslx_read_coo_MM (host only): returns (n, ir, jc, vv) numpy arrays."""
    lib = load()
    coo = CooMat()
    rc = lib.evslx_read_coo_MM(os.fsencode(path), idxin, idxout, C.byref(coo))
    if rc != 0:
        raise EvslError(f"evslx_read_coo_MM returned {rc}: {(lib.evslx_last_error() or b'').decode()}")
    m = coo.nnz
    out = (coo.nrows,
           np.ctypeslib.as_array(coo.ir, (m,)).copy() if m else np.zeros(0, np.int32),
           np.ctypeslib.as_array(coo.jc, (m,)).copy() if m else np.zeros(0, np.int32),
           np.ctypeslib.as_array(coo.vv, (m,)).copy() if m else np.zeros(0))
    lib.free_coo(C.byref(coo))
    return out


def coo_to_csr_host(n, ir, jc, vv, cooidx=0):
    """cooMat_to_csrMat (host only): returns (ia, ja, a)."""
    lib = load()
    ir = np.ascontiguousarray(ir, dtype=np.int32)
    jc = np.ascontiguousarray(jc, dtype=np.int32)
    vv = np.ascontiguousarray(vv, dtype=np.float64)
    coo = CooMat(nrows=n, ncols=n, nnz=len(ir), ir=_i(ir), jc=_i(jc), vv=_d(vv))
    csr = CsrMat()
    rc = lib.cooMat_to_csrMat(cooidx, C.byref(coo), C.byref(csr))
    if rc != 0:
        raise EvslError(f"cooMat_to_csrMat returned {rc}")
    nnz = csr.ia[n]
    out = (np.ctypeslib.as_array(csr.ia, (n + 1,)).copy(),
           np.ctypeslib.as_array(csr.ja, (nnz,)).copy() if nnz else np.zeros(0, np.int32),
           np.ctypeslib.as_array(csr.a, (nnz,)).copy() if nnz else np.zeros(0))
    lib.free_csr(C.byref(csr))
    return out


def simpson(xi, yi):
    """simpson (host only): cumulative integral of yi over xi."""
    lib = load()
    xi = np.ascontiguousarray(xi, dtype=np.float64)
    y = np.array(yi, dtype=np.float64)
    lib.simpson(_d(xi), _d(y), len(y))
    return y


def spslicer2(xi, yi, n_int):
    """spslicer2 (host only): slice boundaries from a DOS curve (yi is not
    modified; the library integrates a copy)."""
    lib = load()
    xi = np.ascontiguousarray(xi, dtype=np.float64)
    y = np.array(yi, dtype=np.float64)
    sli = np.zeros(n_int + 1)
    lib.spslicer2(_d(xi), _d(y), n_int, len(y), _d(sli))
    return sli


def exdos(vals, npts, intv):
    """exDOS (host only): (rc, x, y) for known eigenvalues."""
    lib = load()
    v = np.ascontiguousarray(vals, dtype=np.float64)
    iv = np.ascontiguousarray(intv, dtype=np.float64)
    x, y = np.zeros(npts), np.zeros(npts)
    rc = lib.exDOS(_d(v), len(v), npts, _d(x), _d(y), _d(iv))
    return rc, x, y


def load():
    """Load libevsl_b200.so (raises if it is missing)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `make -C evsl_b200/csrc` "
                          "(or __graft_entry__.build())")
    lib = C.CDLL(path, mode=C.RTLD_LOCAL)
    sig = {
        "EVSLStart": ([], C.c_int),
        "EVSLFinish": ([], C.c_int),
        "SetAMatrix": ([C.POINTER(CsrMat)], C.c_int),
        "SetAMatrix_device_csr": ([C.POINTER(CsrMat)], C.c_int),
        "SetAMatvec": ([C.c_int, C.c_void_p, C.c_void_p], C.c_int),
        "set_pol_def": ([C.POINTER(PolParams)], None),
        "find_pol": ([_dp, C.POINTER(PolParams)], C.c_int),
        "free_pol": ([C.POINTER(PolParams)], None),
        "ChebAv": ([C.POINTER(PolParams), C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
        "ChebLanNr": ([_dp, C.c_int, C.c_double, C.c_void_p, C.POINTER(PolParams), _ip,
                       C.POINTER(_dp), C.POINTER(C.c_void_p), C.POINTER(_dp), C.c_void_p], C.c_int),
        "ChebLanTr": ([C.c_int, C.c_int, _dp, C.c_int, C.c_double, C.c_void_p, C.POINTER(PolParams), _ip,
                       C.POINTER(_dp), C.POINTER(C.c_void_p), C.POINTER(_dp), C.c_void_p], C.c_int),
        "kpmdos": ([C.c_int, C.c_int, C.c_int, _dp, _dp, _dp], C.c_int),
        "LanBounds": ([C.c_int, C.c_void_p, _dp, _dp], C.c_int),
        "evslx_chebav_block": ([C.POINTER(PolParams), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
        "ChebSI": ([C.c_int, _dp, C.c_int, C.c_double, C.c_void_p, C.POINTER(PolParams), _ip, C.POINTER(_dp),
                    C.POINTER(C.c_void_p), C.POINTER(_dp), C.c_void_p], C.c_int),
        "LanTrbounds": ([C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int, _dp, _dp, C.c_void_p], C.c_int),
        "spslicer": ([_dp, _dp, C.c_int, _dp, C.c_int, C.c_int], C.c_int),
        "dampcf": ([C.c_int, C.c_int, _dp], C.c_int),
        "_evsl_Malloc_device": ([C.c_size_t], C.c_void_p),
        "_evsl_Free_device": ([C.c_void_p], None),
        "_evsl_Free": ([C.c_void_p], None),
        "evsl_memcpy_host_to_device": ([C.c_void_p, C.c_void_p, C.c_size_t], None),
        "evsl_memcpy_device_to_host": ([C.c_void_p, C.c_void_p, C.c_size_t], None),
        "rand_double_device": ([C.c_int, C.c_void_p], None),
        "evslx_last_error": ([], C.c_char_p),
        "evslx_set_seed": ([C.c_uint64], C.c_int),
        "evslx_get_draw": ([], C.c_uint64),
        "evslx_kpmdos_probes": ([C.c_int, C.c_int, C.c_int, _dp, C.c_void_p, _dp, _dp], C.c_int),
        "evslx_kpmdos_probes_noalloc": ([C.c_int, C.c_int, C.c_int, _dp, C.c_void_p, _dp, _dp], C.c_int),
        "evslx_set_spmv_kernel": ([C.c_int], C.c_int),
        "evslx_kpm_dots": ([C.c_int, C.c_int, _dp, C.c_void_p, _dp], C.c_int),
        "evslx_kpm_accumulate": ([C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp], C.c_int),
        "evslx_rand_device_draws": ([C.c_int, C.c_int, C.c_uint64, C.c_void_p], C.c_int),
        "evslx_get_spmv_kernel": ([], C.c_int),
        "evslx_matvec": ([C.c_void_p, C.c_void_p], C.c_int),
        "evslx_matvec_cols": ([C.c_int, C.c_void_p, C.c_void_p], C.c_int),
        "evslx_problem_info": ([_ip, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)], C.c_int),
        "evslx_launch_count": ([], C.c_uint64),
        "evslx_last_kpm_seconds": ([], C.c_double),
        "evsl_timer": ([], C.c_double),
        "evslx_stream": ([], C.c_void_p),
        "evslx_filter_profile": ([C.c_int], C.c_int),
        "evslx_filter_stats": ([_dp, _dp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)], C.c_int),
        "StatsReset": ([], None),
        "evslx_last_solve_info": ([_ip, _ip], C.c_int),
        "evslx_set_filter_persistent": ([C.c_int], C.c_int),
        "evslx_set_async_tests": ([C.c_int], C.c_int),
        "evslx_set_filter_block": ([C.c_int], C.c_int),
        "evslx_set_filter_rows_per_thread": ([C.c_int], C.c_int),
        "evslx_set_matrix_compression": ([C.c_int], C.c_int),
        "evslx_matrix_storage": ([_ip, _ip], C.c_int),
        "evslx_set_sell_sigma": ([C.c_int], C.c_int),
        "evslx_set_wait_limit": ([C.c_ulonglong], C.c_int),
        "evslx_set_panel_filter": ([C.c_int, C.c_int, C.c_int], C.c_int),
        "evslx_matrix_panel_layout": ([C.c_int, _ip, _ip, C.POINTER(C.c_longlong)], C.c_int),
        "evslx_matrix_sell_layout": ([_ip, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)], C.c_int),
        "evslx_read_coo_MM": ([C.c_char_p, C.c_int, C.c_int, C.POINTER(CooMat)], C.c_int),
        "evslx_coo_to_csr_device": ([C.c_int, C.POINTER(CooMat), C.c_int, C.POINTER(CsrMat)], C.c_int),
        "cooMat_to_csrMat": ([C.c_int, C.POINTER(CooMat), C.POINTER(CsrMat)], C.c_int),
        "free_coo": ([C.POINTER(CooMat)], None),
        "free_csr": ([C.POINTER(CsrMat)], None),
        "evsl_free_csr_gpu": ([C.POINTER(CsrMat)], None),
        "LanDos": ([C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp], C.c_int),
        "spslicer2": ([_dp, _dp, C.c_int, C.c_int, _dp], None),
        "simpson": ([_dp, _dp, C.c_int], None),
        "exDOS": ([_dp, C.c_int, C.c_int, _dp, _dp, _dp], C.c_int),
        "evslx_matrix_create": ([C.POINTER(CsrMat), C.c_int], C.c_void_p),
        "evslx_matrix_free": ([C.c_void_p], None),
        "evslx_matrix_device_bytes": ([C.c_void_p], C.c_longlong),
        "evslx_engine_create": ([C.c_int, C.c_size_t, C.c_int, C.c_int], C.c_void_p),
        "evslx_engine_free": ([C.c_void_p], None),
        "evslx_engine_submit_slice": ([C.c_void_p, C.c_void_p, _dp, C.POINTER(PolParams), C.c_int, C.c_double,
                                       C.c_void_p, C.c_int, C.c_uint64], C.c_int),
        "evslx_engine_submit_kpm": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, _dp, C.c_uint64,
                                     C.c_uint64], C.c_int),
        "evslx_engine_step": ([C.c_void_p], C.c_int),
        "evslx_engine_run": ([C.c_void_p], C.c_int),
        "evslx_engine_pending": ([C.c_void_p], C.c_int),
        "evslx_engine_bytes_in_use": ([C.c_void_p], C.c_size_t),
        "evslx_engine_pop_result": ([C.c_void_p, C.POINTER(EvslxResult)], C.c_int),
        "evslx_result_free": ([C.POINTER(EvslxResult)], None),
        "evslx_engine_use_graphs": ([C.c_void_p, C.c_int], None),
        "evslx_engine_use_batch": ([C.c_void_p, C.c_int, C.c_int], None),
        "evslx_set_batch_persistent": ([C.c_int], C.c_int),
        "evslx_engine_use_batch_ops": ([C.c_void_p, C.c_int], None),
        "evslx_engine_phase_times": ([C.c_void_p, _dp], None),
        "evslx_engine_batched_columns": ([C.c_void_p], C.c_uint64),
        "evslx_set_mixed_min_rows": ([C.c_int], None),
        "evslx_set_filter_variant": ([C.c_int], C.c_int),
        "evslx_set_split_range_bytes": ([C.c_longlong], C.c_int),
        "evslx_set_l2_resident": ([C.c_int], C.c_int),
        "evslx_set_row_patterns": ([C.c_int], C.c_int),
        "evslx_row_pattern_count": ([], C.c_int),
        "evslx_set_filter_kernel": ([C.c_int], C.c_int),
        "evslx_filter_kernel": ([C.POINTER(C.c_double)], C.c_int),
        "evslx_filter_kernel_grid": ([], C.c_int),
        "evslx_set_filter_wave": ([C.c_int], C.c_int),
        "evslx_get_filter_variant": ([], C.c_int),
        "evslx_tuned_filter_variant": ([C.c_int, C.c_int], C.c_int),
        "evslx_engine_plan_builds": ([C.c_void_p], C.c_uint64),
        "evslx_engine_group_widths": ([C.c_void_p, C.POINTER(C.c_uint64)], None),
        "evslx_chebav_multi": ([C.c_int, C.POINTER(PolParams), C.c_void_p, C.c_void_p, C.c_int], C.c_int),
        "evslx_ChebLanNr_batch": ([C.c_int, _dp, C.c_int, C.c_double, C.c_void_p, C.POINTER(PolParams), C.c_int,
                                   _ip, C.POINTER(_dp), C.POINTER(C.c_void_p), C.POINTER(_dp)], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _LIB = lib
    return lib


class EvslStat(C.Structure):
    """Layout of the reference's timing statistics (INC/struct.h:223-253),
    the library's exported `evslstat`."""
    _fields_ = ([(f, C.c_double) for f in ("t_setBsv", "t_setASigBsv", "t_iter", "t_polAv", "t_reorth",
                                           "t_siorth", "t_ritz", "t_eig", "t_mvA", "t_mvB", "t_svB", "t_svLT",
                                           "t_svASigB", "t_blas", "t_ratAv")] +
                [(f, C.c_size_t) for f in ("n_mvA", "n_mvB", "n_svB", "n_svLT", "n_svASigB", "n_polAv", "n_ratAv",
                                           "alloced", "alloced_total", "alloced_max")])


class DeviceBuffer:
    """A block of device memory owned by the library allocator."""

    def __init__(self, lib, nbytes, ptr=None, owned=True):
        self.lib = lib
        self.nbytes = int(nbytes)
        self.ptr = ptr if ptr is not None else lib._evsl_Malloc_device(max(self.nbytes, 1))
        if not self.ptr:
            raise EvslError(f"device allocation of {nbytes} bytes failed")
        self.owned = owned

    @classmethod
    def from_host(cls, lib, arr):
        arr = np.ascontiguousarray(arr)
        buf = cls(lib, arr.nbytes)
        lib.evsl_memcpy_host_to_device(buf.ptr, arr.ctypes.data, arr.nbytes)
        return buf

    def to_host(self, dtype=np.float64, shape=None):
        out = np.empty(self.nbytes // np.dtype(dtype).itemsize, dtype=dtype)
        self.lib.evsl_memcpy_device_to_host(out.ctypes.data, self.ptr, out.nbytes)
        return out if shape is None else out.reshape(shape)

    def free(self):
        if self.owned and self.ptr:
            self.lib._evsl_Free_device(self.ptr)
        self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Matrix:
    """A resident device matrix (evslx_matrix) owned by this object."""

    def __init__(self, lib, ia, ja, a):
        self.lib = lib
        ia = np.ascontiguousarray(ia, dtype=np.int32)
        ja = np.ascontiguousarray(ja, dtype=np.int32)
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.n = len(ia) - 1
        m = CsrMat(owndata=0, nrows=self.n, ncols=self.n, nnz=int(ia[-1]), ia=_i(ia), ja=_i(ja), a=_d(a))
        self.ptr = lib.evslx_matrix_create(C.byref(m), 0)
        if not self.ptr:
            raise EvslError(f"evslx_matrix_create failed: {(lib.evslx_last_error() or b'').decode()}")

    def device_bytes(self):
        return self.lib.evslx_matrix_device_bytes(self.ptr)

    def free(self):
        if self.ptr:
            self.lib.evslx_matrix_free(self.ptr)
        self.ptr = None


class Engine:
    """Continuous-batching request engine (evslx_engine)."""

    def __init__(self, lib, max_slots, hbm_budget=0, precision=PREC_FP64, keep_vectors=False):
        self.lib = lib
        self.ptr = lib.evslx_engine_create(max_slots, hbm_budget, precision, 1 if keep_vectors else 0)
        self._info = {}
        if not self.ptr:
            raise EvslError(f"evslx_engine_create failed: {(lib.evslx_last_error() or b'').decode()}")

    def _check(self, rc, what):
        if rc != 0:
            raise EvslError(f"{what} returned {rc}: {(self.lib.evslx_last_error() or b'').decode()}")

    def submit_slice(self, M, intv, pol, maxit, tol, vinit, tag):
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        v = np.ascontiguousarray(vinit, dtype=np.float64)
        self._check(self.lib.evslx_engine_submit_slice(self.ptr, M.ptr, _d(iv), C.byref(pol), maxit, tol,
                                                       v.ctypes.data, 0, tag), "evslx_engine_submit_slice")
        self._info[tag] = {"n": M.n}

    def submit_kpm(self, M, Mdeg, damping, nvec, intv, seed, tag):
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        self._check(self.lib.evslx_engine_submit_kpm(self.ptr, M.ptr, Mdeg, damping, nvec, _d(iv), seed, tag),
                    "evslx_engine_submit_kpm")
        self._info[tag] = {"n": M.n, "Mdeg": Mdeg}

    def step(self):
        rc = self.lib.evslx_engine_step(self.ptr)
        if rc < 0:
            self._check(rc, "evslx_engine_step")
        return rc

    def run(self):
        self._check(self.lib.evslx_engine_run(self.ptr), "evslx_engine_run")

    def use_batch_ops(self, on):
        """The slots' Lanczos vector operations in one launch per operation
        (True, default) or per slot (False)."""
        self.lib.evslx_engine_use_batch_ops(self.ptr, 1 if on else 0)

    def phase_times(self):
        """Host seconds per step phase: filter issue, Lanczos issue, scalar wait,
        host part, retirement."""
        out = np.zeros(5)
        self.lib.evslx_engine_phase_times(self.ptr, _d(out))
        return dict(zip(("filter_issue", "lanczos_issue", "scalar_wait", "host", "retire"), out.tolist()))

    def pending(self):
        return self.lib.evslx_engine_pending(self.ptr)

    def bytes_in_use(self):
        return self.lib.evslx_engine_bytes_in_use(self.ptr)

    def use_batch(self, on, max_rows=0):
        self.lib.evslx_engine_use_batch(self.ptr, 1 if on else 0, int(max_rows))

    def batched_columns(self):
        return int(self.lib.evslx_engine_batched_columns(self.ptr))

    def use_graphs(self, on):
        self.lib.evslx_engine_use_graphs(self.ptr, 1 if on else 0)

    def plan_builds(self):
        return self.lib.evslx_engine_plan_builds(self.ptr)

    def group_widths(self):
        """Filter groups launched so far by block width {1, 2, 4, 8, 16}."""
        out = (C.c_uint64 * 5)()
        self.lib.evslx_engine_group_widths(self.ptr, out)
        return dict(zip((1, 2, 4, 8, 16), (int(x) for x in out)))

    def pop(self):
        """Next result as a dict (None if the result queue is empty)."""
        r = EvslxResult()
        if not self.lib.evslx_engine_pop_result(self.ptr, C.byref(r)):
            return None
        info = self._info.pop(r.tag, {})
        out = {"tag": r.tag, "kind": r.kind, "rc": r.rc, "nev": r.nev, "ecnt": r.ecnt,
               "lanczos_steps": r.lanczos_steps, "refine_sweeps": r.refine_sweeps,
               "t_submit": r.t_submit, "t_start": r.t_start, "t_finish": r.t_finish}
        m = r.nev
        out["lam"] = np.ctypeslib.as_array(r.lam, (m,)).copy() if m and r.lam else np.zeros(0)
        out["res"] = np.ctypeslib.as_array(r.res, (m,)).copy() if m and r.res else np.zeros(0)
        out["mu"] = np.ctypeslib.as_array(r.mu, (info["Mdeg"] + 1,)).copy() if r.mu and "Mdeg" in info else None
        out["Y"] = None
        if r.Y and m:
            Y = np.empty((m, info["n"]))
            self.lib.evsl_memcpy_device_to_host(Y.ctypes.data, r.Y, Y.nbytes)
            out["Y"] = Y
        self.lib.evslx_result_free(C.byref(r))
        return out

    def free(self):
        if self.ptr:
            self.lib.evslx_engine_free(self.ptr)
        self.ptr = None


class Library:
    """One EVSL session (EVSLStart ... EVSLFinish) on the current GPU."""

    def __init__(self):
        self.lib = load()
        self._check(self.lib.EVSLStart(), "EVSLStart")
        self.n = 0
        self._csr = None
        self._keep = None

    # -- errors ------------------------------------------------------------
    def last_error(self) -> str:
        return (self.lib.evslx_last_error() or b"").decode(errors="replace")

    def _check(self, rc, what):
        if rc != 0:
            raise EvslError(f"{what} returned {rc}: {self.last_error()}")

    def finish(self):
        self._check(self.lib.EVSLFinish(), "EVSLFinish")

    # -- matrix ------------------------------------------------------------
    def set_csr(self, ia, ja, a):
        """SetAMatrix with a host CSR (uploaded to the device once)."""
        ia = np.ascontiguousarray(ia, dtype=np.int32)
        ja = np.ascontiguousarray(ja, dtype=np.int32)
        a = np.ascontiguousarray(a, dtype=np.float64)
        n = len(ia) - 1
        m = CsrMat(owndata=0, nrows=n, ncols=n, nnz=int(ia[-1]), ia=_i(ia), ja=_i(ja), a=_d(a))
        self._keep = (ia, ja, a, m)
        self._check(self.lib.SetAMatrix(C.byref(m)), "SetAMatrix")
        self.n = n

    def set_csr_device(self, ia, ja, a):
        """SetAMatrix_device_csr with the CSR copied to device buffers first."""
        ia = np.ascontiguousarray(ia, dtype=np.int32)
        ja = np.ascontiguousarray(ja, dtype=np.int32)
        a = np.ascontiguousarray(a, dtype=np.float64)
        n = len(ia) - 1
        bufs = [DeviceBuffer.from_host(self.lib, x) for x in (ia, ja, a)]
        m = CsrMat(owndata=0, nrows=n, ncols=n, nnz=int(ia[-1]), ia=C.cast(bufs[0].ptr, _ip),
                   ja=C.cast(bufs[1].ptr, _ip), a=C.cast(bufs[2].ptr, _dp))
        self._keep = (bufs, m)
        self._check(self.lib.SetAMatrix_device_csr(C.byref(m)), "SetAMatrix_device_csr")
        self.n = n

    def coo_to_csr_device(self, n, ir, jc, vv, cooidx=0, coo_on_device=False):
        """evslx_coo_to_csr_device: returns the device csrMat (owned by the
        caller; release with free_csr_device)."""
        ir = np.ascontiguousarray(ir, dtype=np.int32)
        jc = np.ascontiguousarray(jc, dtype=np.int32)
        vv = np.ascontiguousarray(vv, dtype=np.float64)
        keep = None
        if coo_on_device:
            keep = [DeviceBuffer.from_host(self.lib, x) for x in (ir, jc, vv)]
            coo = CooMat(nrows=n, ncols=n, nnz=len(ir), ir=C.cast(keep[0].ptr, _ip), jc=C.cast(keep[1].ptr, _ip),
                         vv=C.cast(keep[2].ptr, _dp))
        else:
            coo = CooMat(nrows=n, ncols=n, nnz=len(ir), ir=_i(ir), jc=_i(jc), vv=_d(vv))
        csr = CsrMat()
        self._check(self.lib.evslx_coo_to_csr_device(cooidx, C.byref(coo), 1 if coo_on_device else 0, C.byref(csr)),
                    "evslx_coo_to_csr_device")
        del keep
        return csr

    def csr_device_to_host(self, csr):
        n, nnz = csr.nrows, csr.nnz
        ia = np.zeros(n + 1, np.int32)
        ja = np.zeros(max(nnz, 1), np.int32)
        a = np.zeros(max(nnz, 1))
        self.lib.evsl_memcpy_device_to_host(ia.ctypes.data, C.cast(csr.ia, C.c_void_p), ia.nbytes)
        if nnz:
            self.lib.evsl_memcpy_device_to_host(ja.ctypes.data, C.cast(csr.ja, C.c_void_p), 4 * nnz)
            self.lib.evsl_memcpy_device_to_host(a.ctypes.data, C.cast(csr.a, C.c_void_p), 8 * nnz)
        return ia, ja[:nnz], a[:nnz]

    def free_csr_device(self, csr):
        self.lib.evsl_free_csr_gpu(C.byref(csr))

    def set_coo(self, n, ir, jc, vv, cooidx=0, coo_on_device=False):
        """Device COO -> CSR, then SetAMatrix_device_csr on the result (kept
        alive with the session)."""
        csr = self.coo_to_csr_device(n, ir, jc, vv, cooidx, coo_on_device)
        self._keep = (csr,)
        self._check(self.lib.SetAMatrix_device_csr(C.byref(csr)), "SetAMatrix_device_csr")
        self.n = n
        return csr

    def set_filter_wave(self, on):
        self._check(self.lib.evslx_set_filter_wave(1 if on else 0), "evslx_set_filter_wave")

    def set_row_patterns(self, on):
        """Use (default) or stop using the row-pattern dictionary of the stored matrix."""
        self._check(self.lib.evslx_set_row_patterns(1 if on else 0), "evslx_set_row_patterns")

    def row_pattern_count(self):
        """Distinct row patterns of the registered matrix (0: no dictionary)."""
        return int(self.lib.evslx_row_pattern_count())

    FILTER_KERNELS = ("sell-loop", "sell-unrolled", "pattern-global-unrolled", "pattern-global-loop",
                      "pattern-constant-loop", "pattern-constant-unrolled", "pattern-constant-rowdesc", "panel")

    def set_filter_kernel(self, variant):
        """Force a single-vector filter kernel (index or name), or -1/None for timed selection."""
        if variant is None:
            variant = -1
        if isinstance(variant, str):
            variant = self.FILTER_KERNELS.index(variant)
        self._check(self.lib.evslx_set_filter_kernel(int(variant)), "evslx_set_filter_kernel")

    def filter_kernel(self):
        """(chosen variant or -1, {variant name: measured us per degree step}) of the registered matrix."""
        us = (C.c_double * 8)()
        v = int(self.lib.evslx_filter_kernel(us))
        return v, {self.FILTER_KERNELS[i]: us[i] for i in range(8) if us[i] > 0}

    def filter_kernel_grid(self):
        """Blocks per degree step chosen with the filter kernel (0: one row per thread)."""
        return int(self.lib.evslx_filter_kernel_grid())

    def set_l2_resident(self, on):
        self._check(self.lib.evslx_set_l2_resident(1 if on else 0), "evslx_set_l2_resident")

    def set_async_tests(self, on):
        """ChebLanNr's convergence tests on a side stream (default) or waited for."""
        self._check(self.lib.evslx_set_async_tests(1 if on else 0), "evslx_set_async_tests")

    def set_filter_persistent(self, on):
        self._check(self.lib.evslx_set_filter_persistent(1 if on else 0), "evslx_set_filter_persistent")

    def set_matrix_compression(self, on):
        self._check(self.lib.evslx_set_matrix_compression(1 if on else 0), "evslx_set_matrix_compression")

    def matrix_storage(self):
        vb, ib = C.c_int(), C.c_int()
        self._check(self.lib.evslx_matrix_storage(C.byref(vb), C.byref(ib)), "evslx_matrix_storage")
        return vb.value, ib.value

    def set_wait_limit(self, polls):
        """Polls before a device-side wait gives up (0: the defaults)."""
        self._check(self.lib.evslx_set_wait_limit(int(polls)), "evslx_set_wait_limit")

    def set_panel_filter(self, on, min_rows=0, max_width=0):
        """Build (default) or skip the column-panel layout of large general matrices."""
        self._check(self.lib.evslx_set_panel_filter(1 if on else 0, int(min_rows), int(max_width)),
                    "evslx_set_panel_filter")

    def matrix_panel_layout(self, fp32=False):
        """(rows per block, panel width, device bytes) of the panel layout (zeros if none)."""
        r, w, b = C.c_int(), C.c_int(), C.c_longlong()
        self._check(self.lib.evslx_matrix_panel_layout(1 if fp32 else 0, C.byref(r), C.byref(w), C.byref(b)),
                    "evslx_matrix_panel_layout")
        return r.value, w.value, b.value

    def set_sell_sigma(self, sigma):
        """SELL-C-sigma row sort window for matrices registered afterwards: -1
        automatic (default), 0 never, or a power of two from 32 to 4096."""
        self._check(self.lib.evslx_set_sell_sigma(int(sigma)), "evslx_set_sell_sigma")

    def matrix_sell_layout(self):
        """(sort window in use or 0, stored slots, slots of the unsorted layout)."""
        sg, st, su = C.c_int(), C.c_longlong(), C.c_longlong()
        self._check(self.lib.evslx_matrix_sell_layout(C.byref(sg), C.byref(st), C.byref(su)),
                    "evslx_matrix_sell_layout")
        return sg.value, st.value, su.value

    def set_spmv_kernel(self, which):
        self._check(self.lib.evslx_set_spmv_kernel(which), "evslx_set_spmv_kernel")

    def problem_info(self):
        n = C.c_int()
        nnz = C.c_longlong()
        st = C.c_longlong()
        self.lib.evslx_problem_info(C.byref(n), C.byref(nnz), C.byref(st))
        return n.value, nnz.value, st.value

    def matvec(self, x):
        dx = DeviceBuffer.from_host(self.lib, np.asarray(x, dtype=np.float64))
        dy = DeviceBuffer(self.lib, dx.nbytes)
        self._check(self.lib.evslx_matvec(dx.ptr, dy.ptr), "evslx_matvec")
        return dy.to_host()

    def matvec_cols(self, X):
        """Rows of X (m x n) each multiplied by A, in one launch."""
        X = np.ascontiguousarray(np.atleast_2d(X), dtype=np.float64)
        dx = DeviceBuffer.from_host(self.lib, X)
        dy = DeviceBuffer(self.lib, dx.nbytes)
        self._check(self.lib.evslx_matvec_cols(X.shape[0], dx.ptr, dy.ptr), "evslx_matvec_cols")
        return dy.to_host().reshape(X.shape)

    # -- filter --------------------------------------------------------------
    def find_pol(self, intv, *, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=None, deg=0):
        pol = PolParams()
        self.lib.set_pol_def(C.byref(pol))
        pol.damping = damping
        pol.thresh_int = thresh_int
        pol.thresh_ext = thresh_ext
        if max_deg is not None:
            pol.max_deg = max_deg
        pol.deg = deg
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        rc = self.lib.find_pol(_d(iv), C.byref(pol))
        if rc != 0:
            raise EvslError(f"find_pol returned {rc}")
        return pol

    def free_pol(self, pol):
        self.lib.free_pol(C.byref(pol))

    def chebav(self, pol, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        dv = DeviceBuffer.from_host(self.lib, v)
        dy = DeviceBuffer(self.lib, v.nbytes)
        dw = DeviceBuffer(self.lib, 3 * v.nbytes)
        self._check(self.lib.ChebAv(C.byref(pol), dv.ptr, dy.ptr, dw.ptr), "ChebAv")
        return dy.to_host()

    def chebav_block(self, pol, V):
        """p(A) applied to the rows of V (ncols x n) with the block filter."""
        V = np.ascontiguousarray(V, dtype=np.float64)
        dv = DeviceBuffer.from_host(self.lib, V)
        dy = DeviceBuffer(self.lib, V.nbytes)
        dw = DeviceBuffer(self.lib, 2 * V.nbytes)
        self._check(self.lib.evslx_chebav_block(C.byref(pol), V.shape[0], dv.ptr, dy.ptr, dw.ptr),
                    "evslx_chebav_block")
        return dy.to_host().reshape(V.shape)

    # -- spectrum bounds -----------------------------------------------------
    def lan_bounds(self, msteps, v):
        """LanBounds on a host start vector (copied to the device)."""
        dv = DeviceBuffer.from_host(self.lib, np.asarray(v, dtype=np.float64))
        lo, hi = C.c_double(), C.c_double()
        self._check(self.lib.LanBounds(msteps, dv.ptr, C.byref(lo), C.byref(hi)), "LanBounds")
        return lo.value, hi.value

    def lan_trbounds(self, lanm, maxit, tol, v, bndtype=1):
        dv = DeviceBuffer.from_host(self.lib, np.asarray(v, dtype=np.float64))
        lo, hi = C.c_double(), C.c_double()
        self._check(self.lib.LanTrbounds(lanm, maxit, tol, dv.ptr, bndtype, C.byref(lo), C.byref(hi), None),
                    "LanTrbounds")
        return lo.value, hi.value

    def chebav_multi(self, pols, X, precision=PREC_FP64):
        """evslx_chebav_multi: rows of X (ncols x n) filtered by pols[c]."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        arr = (PolParams * len(pols))(*pols)
        dx = DeviceBuffer.from_host(self.lib, X)
        dy = DeviceBuffer(self.lib, X.nbytes)
        self._check(self.lib.evslx_chebav_multi(len(pols), arr, dx.ptr, dy.ptr, precision), "evslx_chebav_multi")
        return dy.to_host().reshape(X.shape)

    def cheblan_nr_batch(self, intvs, maxit, tol, vinit, pols, precision=PREC_FP64, want_vectors=True):
        """evslx_ChebLanNr_batch: list of (lam, Y, res) per slice."""
        ns = len(pols)
        iv = np.ascontiguousarray(np.asarray(intvs, dtype=np.float64).reshape(ns * 4))
        arr = (PolParams * ns)(*pols)
        dv = DeviceBuffer.from_host(self.lib, np.asarray(vinit, dtype=np.float64))
        nev = (C.c_int * ns)()
        lam = (_dp * ns)()
        W = (C.c_void_p * ns)()
        res = (_dp * ns)()
        rc = self.lib.evslx_ChebLanNr_batch(ns, _d(iv), maxit, tol, dv.ptr, arr, precision, nev, lam, W, res)
        self._check(rc, "evslx_ChebLanNr_batch")
        return [self._outputs(nev[s], lam[s], W[s], res[s], want_vectors) for s in range(ns)]

    def set_mixed_min_rows(self, rows):
        """Engines created afterwards use the FP32 filter only on matrices
        with at least this many rows."""
        self.lib.evslx_set_mixed_min_rows(int(rows))

    def set_filter_variant(self, v):
        self._check(self.lib.evslx_set_filter_variant(v), "evslx_set_filter_variant")

    def tuned_filter_variant(self, precision, ncols):
        return self.lib.evslx_tuned_filter_variant(precision, ncols)

    def set_batch_persistent(self, on):
        """The engines' batched filter as one persistent launch (True) or one
        launch per degree (False, default)."""
        self._check(self.lib.evslx_set_batch_persistent(1 if on else 0), "evslx_set_batch_persistent")

    def set_split_range_bytes(self, nbytes):
        """Bytes of block rows one column range of filter variant 7 gathers
        from (0: the default)."""
        self._check(self.lib.evslx_set_split_range_bytes(int(nbytes)), "evslx_set_split_range_bytes")

    def matrix(self, ia, ja, a):
        return Matrix(self.lib, ia, ja, a)

    def engine(self, max_slots, hbm_budget=0, precision=PREC_FP64, keep_vectors=False):
        return Engine(self.lib, max_slots, hbm_budget, precision, keep_vectors)

    def lan_dos(self, nvec, msteps, npts, intv):
        """LanDos: returns (xdos, ydos, neig)."""
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        x, y = np.zeros(npts), np.zeros(npts)
        ne = C.c_double()
        self._check(self.lib.LanDos(nvec, msteps, npts, _d(x), _d(y), C.byref(ne), _d(iv)), "LanDos")
        return x, y, ne.value

    # -- DOS / slicing -----------------------------------------------------
    def set_seed(self, seed):
        self.lib.evslx_set_seed(seed)

    def kpmdos(self, Mdeg, damping, nvec, intv):
        mu = np.zeros(Mdeg + 1)
        ec = C.c_double()
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        self._check(self.lib.kpmdos(Mdeg, damping, nvec, _d(iv), _d(mu), C.byref(ec)), "kpmdos")
        return mu, ec.value

    def kpmdos_probes(self, Mdeg, damping, probes, intv):
        """kpmdos with explicit probe vectors (nvec x n host array)."""
        probes = np.ascontiguousarray(np.atleast_2d(probes), dtype=np.float64)
        dp = DeviceBuffer.from_host(self.lib, probes)  # row p = probe p = column p of n x nvec
        mu = np.zeros(Mdeg + 1)
        ec = C.c_double()
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        self._check(self.lib.evslx_kpmdos_probes(Mdeg, damping, probes.shape[0], _d(iv), dp.ptr, _d(mu),
                                                 C.byref(ec)), "evslx_kpmdos_probes")
        return mu, ec.value

    def kpm_dots(self, Mdeg, intv, dprobes, nvec):
        """Raw KPM dot products (Mdeg x nvec) for device probes (DeviceBuffer)."""
        dots = np.zeros((Mdeg, nvec))
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        self._check(self.lib.evslx_kpm_dots(Mdeg, nvec, _d(iv), dprobes.ptr, _d(dots)), "evslx_kpm_dots")
        return dots

    def draw_probes(self, n, first, count):
        """Device probes for draws first .. first+count-1 of the generator."""
        buf = DeviceBuffer(self.lib, 8 * n * count)
        self._check(self.lib.evslx_rand_device_draws(n, count, first, buf.ptr), "evslx_rand_device_draws")
        return buf

    def spslicer(self, mu, intv, n_int, npts):
        sli = np.zeros(n_int + 1)
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        rc = self.lib.spslicer(_d(sli), _d(mu), len(mu) - 1, _d(iv), n_int, npts)
        return rc, sli

    # -- Lanczos -------------------------------------------------------------
    def _outputs(self, m, lam, W, res, want_vectors):
        n = self.n
        if m > 0:
            lam_h = np.ctypeslib.as_array(lam, (m,)).copy()
            res_h = np.ctypeslib.as_array(res, (m,)).copy()
            Y = None
            if want_vectors:
                Y = np.empty((m, n))
                self.lib.evsl_memcpy_device_to_host(Y.ctypes.data, W, Y.nbytes)
        else:
            lam_h, res_h, Y = np.zeros(0), np.zeros(0), (np.zeros((0, n)) if want_vectors else None)
        for p in (lam, res):
            if p:
                self.lib._evsl_Free(C.cast(p, C.c_void_p))
        if W:
            self.lib._evsl_Free_device(W)
        return lam_h, Y, res_h

    def cheblan_nr(self, intv, maxit, tol, vinit, pol, want_vectors=True):
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        dv = DeviceBuffer.from_host(self.lib, np.asarray(vinit, dtype=np.float64))
        nev = C.c_int()
        lam, res = _dp(), _dp()
        W = C.c_void_p()
        rc = self.lib.ChebLanNr(_d(iv), maxit, tol, dv.ptr, C.byref(pol), C.byref(nev), C.byref(lam),
                                C.byref(W), C.byref(res), None)
        self._check(rc, "ChebLanNr")
        return self._outputs(nev.value, lam, W.value, res, want_vectors)

    def cheblan_tr(self, lanm, nev, intv, maxit, tol, vinit, pol, want_vectors=True):
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        dv = DeviceBuffer.from_host(self.lib, np.asarray(vinit, dtype=np.float64))
        nev2 = C.c_int()
        lam, res = _dp(), _dp()
        W = C.c_void_p()
        rc = self.lib.ChebLanTr(lanm, nev, _d(iv), maxit, tol, dv.ptr, C.byref(pol), C.byref(nev2), C.byref(lam),
                                C.byref(W), C.byref(res), None)
        self._check(rc, "ChebLanTr")
        return self._outputs(nev2.value, lam, W.value, res, want_vectors)

    def cheb_si(self, nev, intv, maxit, tol, vinit_block, pol, want_vectors=True):
        """ChebSI with a host start block (nev x n rows = columns of the n x nev block)."""
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        dv = DeviceBuffer.from_host(self.lib, np.ascontiguousarray(vinit_block, dtype=np.float64))
        nevo = C.c_int()
        lam, res = _dp(), _dp()
        W = C.c_void_p()
        self._check(self.lib.ChebSI(nev, _d(iv), maxit, tol, dv.ptr, C.byref(pol), C.byref(nevo), C.byref(lam),
                                    C.byref(W), C.byref(res), None), "ChebSI")
        return self._outputs(nevo.value, lam, W.value, res, want_vectors)

    def launch_count(self):
        return int(self.lib.evslx_launch_count())

    def last_solve_info(self):
        """(Lanczos dimension, Ritz candidates) of the last Lanczos solve."""
        k, c = C.c_int(), C.c_int()
        self.lib.evslx_last_solve_info(C.byref(k), C.byref(c))
        return k.value, c.value

    def stream_handle(self):
        """cudaStream_t of the library (for recording CUDA events on it)."""
        return int(self.lib.evslx_stream() or 0)

    def stats(self):
        """The timing statistics of the last solves (`evslstat`, reset by
        StatsReset) as a dict of its fields."""
        st = EvslStat.in_dll(self.lib, "evslstat")
        return {f: getattr(st, f) for f, _ in EvslStat._fields_}

    def stats_reset(self):
        self.lib.StatsReset()

    def filter_profile(self, enable=True):
        self._check(self.lib.evslx_filter_profile(1 if enable else 0), "evslx_filter_profile")

    def filter_stats(self):
        """(device seconds, algorithmic bytes, kernel launches, filter calls)."""
        sec, byt = C.c_double(), C.c_double()
        la, ca = C.c_uint64(), C.c_uint64()
        self._check(self.lib.evslx_filter_stats(C.byref(sec), C.byref(byt), C.byref(la), C.byref(ca)),
                    "evslx_filter_stats")
        return sec.value, byt.value, int(la.value), int(ca.value)
