"""CPU oracle for EVSL's polynomial-filtered spectrum-slicing path.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py may import this module.  The
shipped library (evsl_b200) never calls it.

Two independent CPU implementations live here:

* ``RefLib`` -- ctypes access to the reference EVSL C library itself, compiled
  from the reference sources by oracle/Makefile into oracle/_ref/ (with the
  rand_double_device hook of oracle/ref_hooks.c so that probe and start
  vectors can be injected).
* A numpy restatement of the same algorithms (``dampcf``, ``find_pol``,
  ``cheb_av``, ``kpmdos``, ``spslicer``, ``cheblan_nr`` ...), each citing the
  reference file:line it follows.  The restatement is pinned against RefLib by
  tests/test_oracle.py and against the committed golden fixtures in
  tests/golden/ (generated from RefLib by tests/golden/make_golden.py).

All reference paths are relative to the EVSL_1.1.1 project directory.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB_PATH = os.path.join(_HERE, "_ref", "libevsl_ref.so")

EVSL_PI = 3.14159265358979323846  # INC/evsl.h:22
DBL_EPS = np.finfo(np.float64).eps
EVSL_DBL_EPS_MULT = 10  # INC/evsl.h:27
ORTH_TOL = 1e-14  # INC/internal_header.h:21
NGS_MAX = 2  # INC/internal_header.h:24


# ---------------------------------------------------------------------------
# ctypes layout of polparams (INC/struct.h:68-98).  The GPU library keeps the
# same layout, so one definition serves both in the harness.
# ---------------------------------------------------------------------------
class PolParams(C.Structure):
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


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class CooMat(C.Structure):
    """cooMat (INC/struct.h:14-21)."""
    _fields_ = [("nrows", C.c_int), ("ncols", C.c_int), ("nnz", C.c_int), ("ir", _ip), ("jc", _ip), ("vv", _dp)]


class CsrMatCPU(C.Structure):
    """csrMat of the reference CPU build (INC/struct.h:29-42 without the
    CUDA-only members)."""
    _fields_ = [("owndata", C.c_int), ("nrows", C.c_int), ("ncols", C.c_int), ("nnz", C.c_int), ("ia", _ip),
                ("ja", _ip), ("a", _dp)]


def _dptr(a):
    return a.ctypes.data_as(_dp)


def _iptr(a):
    return a.ctypes.data_as(_ip)


class RefLib:
    """The reference EVSL CPU build (oracle/_ref/libevsl_ref.so)."""

    _lib = None

    def __init__(self, path: str = REF_LIB_PATH):
        if RefLib._lib is None:
            if not os.path.exists(path):
                raise FileNotFoundError(
                    f"{path} missing: build it with `make -C oracle` where the reference sources exist")
            lib = C.CDLL(path, mode=C.RTLD_LOCAL)
            lib.EVSLStart.restype = C.c_int
            lib.EVSLFinish.restype = C.c_int
            lib.set_pol_def.argtypes = [C.POINTER(PolParams)]
            lib.find_pol.argtypes = [_dp, C.POINTER(PolParams)]
            lib.find_pol.restype = C.c_int
            lib.free_pol.argtypes = [C.POINTER(PolParams)]
            lib.kpmdos.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]
            lib.kpmdos.restype = C.c_int
            lib.spslicer.argtypes = [_dp, _dp, C.c_int, _dp, C.c_int, C.c_int]
            lib.spslicer.restype = C.c_int
            lib.ChebLanNr.argtypes = [_dp, C.c_int, C.c_double, _dp, C.POINTER(PolParams), _ip,
                                      C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp), C.c_void_p]
            lib.ChebLanNr.restype = C.c_int
            lib.ChebLanTr.argtypes = [C.c_int, C.c_int, _dp, C.c_int, C.c_double, _dp,
                                      C.POINTER(PolParams), _ip, C.POINTER(_dp), C.POINTER(_dp),
                                      C.POINTER(_dp), C.c_void_p]
            lib.ChebLanTr.restype = C.c_int
            lib.evslref_set_seed.argtypes = [C.c_uint64]
            lib.evslref_queue_vectors.argtypes = [_dp, C.c_int, C.c_int]
            lib.evslref_queue_vectors.restype = C.c_int
            lib.evslref_queue_remaining.restype = C.c_int
            lib.evslref_lap_csr.argtypes = [C.c_int, C.c_int, C.c_int, _ip, C.POINTER(_ip),
                                            C.POINTER(_ip), C.POINTER(_dp)]
            lib.evslref_lap_csr.restype = C.c_int
            lib.evslref_free.argtypes = [C.c_void_p]
            lib.evslref_exeig.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _dp, C.c_int]
            lib.evslref_exeig.restype = C.c_int
            lib.evslref_set_csr.argtypes = [C.c_int, _ip, _ip, _dp]
            lib.evslref_set_csr.restype = C.c_int
            lib.evslref_matvec.argtypes = [_dp, _dp]
            lib.evslref_chebav.argtypes = [C.POINTER(PolParams), _dp, _dp]
            lib.evslref_chebav.restype = C.c_int
            lib.evslref_slices_nr.argtypes = [C.c_int, _dp, C.c_double, C.c_double, C.c_int, C.c_double,
                                              _dp, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                              _ip, _ip, _dp, _dp, _dp, C.c_int]
            lib.evslref_slices_nr.restype = C.c_double
            lib._evsl_Free.argtypes = [C.c_void_p]
            lib.LanBounds.argtypes = [C.c_int, _dp, _dp, _dp]
            lib.LanBounds.restype = C.c_int
            lib.LanTrbounds.argtypes = [C.c_int, C.c_int, C.c_double, _dp, C.c_int, _dp, _dp, C.c_void_p]
            lib.LanTrbounds.restype = C.c_int
            lib.evslref_chebav_multi.argtypes = [C.POINTER(PolParams), C.c_int, _dp, C.c_int]
            lib.evslref_chebav_multi.restype = C.c_double
            lib.evslref_cheb_si.argtypes = [C.c_int, _dp, C.c_int, C.c_double, _dp, C.POINTER(PolParams), _ip,
                                            C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp)]
            lib.evslref_cheb_si.restype = C.c_int
            lib.read_coo_MM.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(CooMat)]
            lib.read_coo_MM.restype = C.c_int
            lib.cooMat_to_csrMat.argtypes = [C.c_int, C.POINTER(CooMat), C.POINTER(CsrMatCPU)]
            lib.cooMat_to_csrMat.restype = C.c_int
            lib.free_coo.argtypes = [C.POINTER(CooMat)]
            lib.free_csr.argtypes = [C.POINTER(CsrMatCPU)]
            lib.LanDos.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp]
            lib.LanDos.restype = C.c_int
            lib.spslicer2.argtypes = [_dp, _dp, C.c_int, C.c_int, _dp]
            lib.simpson.argtypes = [_dp, _dp, C.c_int]
            lib.exDOS.argtypes = [_dp, C.c_int, C.c_int, _dp, _dp, _dp]
            lib.exDOS.restype = C.c_int
            lib.EVSLStart()
            RefLib._lib = lib
        self.lib = RefLib._lib
        self._keep = None

    # -- matrices --------------------------------------------------------
    def lap_csr(self, nx, ny, nz):
        """CSR arrays of the reference Laplacian (TESTS/COMMON/lapl.c:13)."""
        n = C.c_int()
        ia, ja, a = _ip(), _ip(), _dp()
        rc = self.lib.evslref_lap_csr(nx, ny, nz, C.byref(n), C.byref(ia), C.byref(ja), C.byref(a))
        assert rc == 0
        nn = n.value
        nnz = ia[nn]
        out = (np.ctypeslib.as_array(ia, (nn + 1,)).copy(),
               np.ctypeslib.as_array(ja, (nnz,)).copy(),
               np.ctypeslib.as_array(a, (nnz,)).copy())
        for p in (ia, ja, a):
            self.lib.evslref_free(C.cast(p, C.c_void_p))
        return out

    def exeig(self, nx, ny, nz, a, b):
        """Analytic Laplacian eigenvalues in [a, b] (TESTS/COMMON/lapl.c:79)."""
        cap = nx * ny * nz
        out = np.zeros(cap)
        m = self.lib.evslref_exeig(nx, ny, nz, a, b, _dptr(out), cap)
        return out[:m].copy()

    def set_csr(self, ia, ja, a):
        ia = np.ascontiguousarray(ia, dtype=np.int32)
        ja = np.ascontiguousarray(ja, dtype=np.int32)
        a = np.ascontiguousarray(a, dtype=np.float64)
        self._keep = (ia, ja, a)  # borrowed by the library
        return self.lib.evslref_set_csr(len(ia) - 1, _iptr(ia), _iptr(ja), _dptr(a))

    def matvec(self, x):
        n = len(self._keep[0]) - 1
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(n)
        self.lib.evslref_matvec(_dptr(x), _dptr(y))
        return y

    # -- RNG hook ----------------------------------------------------------
    def set_seed(self, seed):
        self.lib.evslref_set_seed(seed)

    def queue_vectors(self, vecs):
        vecs = np.ascontiguousarray(vecs, dtype=np.float64)
        if vecs.ndim == 1:
            vecs = vecs[None, :]
        return self.lib.evslref_queue_vectors(_dptr(vecs), vecs.shape[0], vecs.shape[1])

    # -- filter --------------------------------------------------------------
    def find_pol(self, intv, *, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=None,
                 deg=0, min_deg=None, intvtol=None):
        pol = PolParams()
        self.lib.set_pol_def(C.byref(pol))
        pol.damping = damping
        pol.thresh_int = thresh_int
        pol.thresh_ext = thresh_ext
        if max_deg is not None:
            pol.max_deg = max_deg
        if min_deg is not None:
            pol.min_deg = min_deg
        if intvtol is not None:
            pol.intvtol = intvtol
        pol.deg = deg
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        rc = self.lib.find_pol(_dptr(iv), C.byref(pol))
        return rc, pol

    def pol_dict(self, pol):
        mu = np.ctypeslib.as_array(pol.mu, (pol.deg + 1,)).copy() if pol.mu else None
        return dict(type=pol.type, deg=pol.deg, cc=pol.cc, dd=pol.dd, gam=pol.gam, bar=pol.bar, mu=mu)

    def free_pol(self, pol):
        self.lib.free_pol(C.byref(pol))

    def chebav(self, pol, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        y = np.zeros_like(v)
        self.lib.evslref_chebav(C.byref(pol), _dptr(v), _dptr(y))
        return y

    # -- DOS / slicing -------------------------------------------------------
    def kpmdos(self, Mdeg, damping, probes, intv):
        """kpmdos (SRC/spslice.c:29) fed the given probe vectors (nvec x n)."""
        probes = np.atleast_2d(probes)
        self.queue_vectors(probes)
        mu = np.zeros(Mdeg + 1)
        ecnt = C.c_double()
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        rc = self.lib.kpmdos(Mdeg, damping, probes.shape[0], _dptr(iv), _dptr(mu), C.byref(ecnt))
        self.queue_vectors(np.zeros((0, 1)))
        return rc, mu, ecnt.value

    def spslicer(self, mu, intv, n_int, npts):
        sli = np.zeros(n_int + 1)
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        rc = self.lib.spslicer(_dptr(sli), _dptr(mu), len(mu) - 1, _dptr(iv), n_int, npts)
        return rc, sli

    # -- Lanczos ---------------------------------------------------------------
    def cheblan_nr(self, intv, maxit, tol, vinit, pol):
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        v0 = np.ascontiguousarray(vinit, dtype=np.float64)
        nev = C.c_int()
        lam, W, res = _dp(), _dp(), _dp()
        rc = self.lib.ChebLanNr(_dptr(iv), maxit, tol, _dptr(v0), C.byref(pol), C.byref(nev),
                                C.byref(lam), C.byref(W), C.byref(res), None)
        return rc, self._take(nev.value, lam, W, res, len(v0))

    def cheblan_tr(self, lanm, nev, intv, maxit, tol, vinit, pol):
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        v0 = np.ascontiguousarray(vinit, dtype=np.float64)
        nev2 = C.c_int()
        lam, W, res = _dp(), _dp(), _dp()
        rc = self.lib.ChebLanTr(lanm, nev, _dptr(iv), maxit, tol, _dptr(v0), C.byref(pol),
                                C.byref(nev2), C.byref(lam), C.byref(W), C.byref(res), None)
        return rc, self._take(nev2.value, lam, W, res, len(v0))

    def cheb_si(self, nev, intv, maxit, tol, vinit_block, pol):
        """Reference ChebSI (SRC/chebsi.c:39) with start block vinit_block
        (nev x n: row j is column j of the n x nev block)."""
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        v0 = np.ascontiguousarray(vinit_block, dtype=np.float64)
        nevo = C.c_int()
        lam, W, res = _dp(), _dp(), _dp()
        rc = self.lib.evslref_cheb_si(nev, _dptr(iv), maxit, tol, _dptr(v0), C.byref(pol), C.byref(nevo),
                                      C.byref(lam), C.byref(W), C.byref(res))
        return rc, self._take(nevo.value, lam, W, res, v0.shape[1])

    def _take(self, m, lam, W, res, n):
        if m > 0:
            out = (np.ctypeslib.as_array(lam, (m,)).copy(),
                   np.ctypeslib.as_array(W, (m * n,)).copy().reshape(m, n),
                   np.ctypeslib.as_array(res, (m,)).copy())
        else:
            out = (np.zeros(0), np.zeros((0, n)), np.zeros(0))
        for p in (lam, W, res):
            if p:
                self.lib._evsl_Free(C.cast(p, C.c_void_p))
        return out

    def lan_bounds(self, msteps, v):
        """LanBounds (SRC/lanbounds.c:21)."""
        v = np.ascontiguousarray(v, dtype=np.float64)
        lo, hi = C.c_double(), C.c_double()
        rc = self.lib.LanBounds(msteps, _dptr(v), C.byref(lo), C.byref(hi))
        return rc, lo.value, hi.value

    def lan_trbounds(self, lanm, maxit, tol, v, bndtype):
        """LanTrbounds (SRC/lanTrbounds.c:35)."""
        v = np.ascontiguousarray(v, dtype=np.float64)
        lo, hi = C.c_double(), C.c_double()
        rc = self.lib.LanTrbounds(lanm, maxit, tol, _dptr(v), bndtype, C.byref(lo), C.byref(hi), None)
        return rc, lo.value, hi.value

    # -- matrix input (TESTS/COMMON/io.c:115, SRC/spmat.c:160) ------------------
    def read_coo_mm(self, path, idxin=1, idxout=0):
        """Reference read_coo_MM: (rc, n, ir, jc, vv)."""
        coo = CooMat()
        rc = self.lib.read_coo_MM(os.fsencode(path), idxin, idxout, C.byref(coo))
        if rc != 0:
            return rc, 0, None, None, None
        m = coo.nnz
        out = (rc, coo.nrows, np.ctypeslib.as_array(coo.ir, (m,)).copy(),
               np.ctypeslib.as_array(coo.jc, (m,)).copy(), np.ctypeslib.as_array(coo.vv, (m,)).copy())
        self.lib.free_coo(C.byref(coo))
        return out

    def coo_to_csr(self, n, ir, jc, vv, cooidx=0):
        """Reference cooMat_to_csrMat (with its sortrow): (ia, ja, a)."""
        ir = np.ascontiguousarray(ir, dtype=np.int32)
        jc = np.ascontiguousarray(jc, dtype=np.int32)
        vv = np.ascontiguousarray(vv, dtype=np.float64)
        coo = CooMat(nrows=n, ncols=n, nnz=len(ir), ir=_iptr(ir), jc=_iptr(jc), vv=_dptr(vv))
        csr = CsrMatCPU()
        self.lib.cooMat_to_csrMat(cooidx, C.byref(coo), C.byref(csr))
        nnz = csr.ia[n]
        out = (np.ctypeslib.as_array(csr.ia, (n + 1,)).copy(), np.ctypeslib.as_array(csr.ja, (nnz,)).copy(),
               np.ctypeslib.as_array(csr.a, (nnz,)).copy())
        self.lib.free_csr(C.byref(csr))
        return out

    # -- Lanczos DOS (SRC/landos.c:37, SRC/spslice2.c:25, SRC/exDOS.c:17) -------
    def lan_dos(self, nvec, msteps, npts, intv):
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        x, y = np.zeros(npts), np.zeros(npts)
        ne = C.c_double()
        rc = self.lib.LanDos(nvec, msteps, npts, _dptr(x), _dptr(y), C.byref(ne), _dptr(iv))
        return rc, x, y, ne.value

    def spslicer2(self, x, y, n_int):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.array(y, dtype=np.float64)
        sli = np.zeros(n_int + 1)
        self.lib.spslicer2(_dptr(x), _dptr(y), n_int, len(y), _dptr(sli))
        return sli

    def simpson(self, x, y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.array(y, dtype=np.float64)
        self.lib.simpson(_dptr(x), _dptr(y), len(y))
        return y

    def exdos(self, vals, npts, intv):
        v = np.ascontiguousarray(vals, dtype=np.float64)
        iv = np.ascontiguousarray(intv, dtype=np.float64)
        x, y = np.zeros(npts), np.zeros(npts)
        rc = self.lib.exDOS(_dptr(v), len(v), npts, _dptr(x), _dptr(y), _dptr(iv))
        return rc, x, y

    def chebav_multi(self, pol, deg, v, nthreads):
        """Wall seconds of `nthreads` concurrent reference ChebAv calls
        truncated to `deg` degrees (CPU baseline sampler)."""
        v = np.ascontiguousarray(v, dtype=np.float64)
        return self.lib.evslref_chebav_multi(C.byref(pol), deg, _dptr(v), nthreads)

    def slices_nr(self, sli, lmin, lmax, maxit, tol, vinit, *, damping=2, thresh_int=0.8,
                  thresh_ext=0.2, max_deg=10000, nthreads=0, evcap=4096):
        sli = np.ascontiguousarray(sli, dtype=np.float64)
        ns = len(sli) - 1
        v0 = np.ascontiguousarray(vinit, dtype=np.float64)
        nev = np.zeros(ns, dtype=np.int32)
        deg = np.zeros(ns, dtype=np.int32)
        secs = np.zeros(ns)
        ev = np.zeros(ns * evcap)
        rs = np.zeros(ns * evcap)
        wall = self.lib.evslref_slices_nr(ns, _dptr(sli), lmin, lmax, maxit, tol, _dptr(v0), damping,
                                          thresh_int, thresh_ext, max_deg, nthreads, _iptr(nev),
                                          _iptr(deg), _dptr(secs), _dptr(ev), _dptr(rs), evcap)
        evals = [np.sort(ev[s * evcap:s * evcap + nev[s]]) for s in range(ns)]
        resid = [rs[s * evcap:s * evcap + nev[s]].copy() for s in range(ns)]
        return dict(wall=wall, nev=nev, deg=deg, seconds=secs, evals=evals, resids=resid)


# ===========================================================================
# numpy restatement
# ===========================================================================

def lap_csr(nx, ny, nz):
    """2-D/3-D Dirichlet Laplacian in CSR, rows sorted by column.

    Restates lapgen (TESTS/COMMON/lapl.c:13-65) followed by cooMat_to_csrMat +
    sortrow (SRC/spmat.c:160-195, :67-85): diagonal 4 (2-D) or 6 (3-D),
    off-diagonals -1, x fastest.
    """
    n = nx * ny * nz
    idx = np.arange(n, dtype=np.int64)
    k = idx // (nx * ny)
    i = (idx - k * nx * ny) // nx
    j = idx - k * nx * ny - i * nx
    rows, cols, vals = [], [], []
    for mask, off in ((k > 0, -nx * ny), (k < nz - 1, nx * ny), (i > 0, -nx), (i < ny - 1, nx),
                      (j > 0, -1), (j < nx - 1, 1)):
        r = idx[mask]
        rows.append(r)
        cols.append(r + off)
        vals.append(np.full(len(r), -1.0))
    rows.append(idx)
    cols.append(idx)
    vals.append(np.full(n, 6.0 if nz > 1 else 4.0))
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    vals = np.concatenate(vals)
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    ia = np.zeros(n + 1, dtype=np.int64)
    np.add.at(ia, rows + 1, 1)
    ia = np.cumsum(ia)
    return ia.astype(np.int32), cols.astype(np.int32), vals


def exeiglap3(nx, ny, nz, a, b):
    """Analytic Laplacian eigenvalues in [a, b], sorted (TESTS/COMMON/lapl.c:79-109)."""
    tx = np.sin(np.arange(1, nx + 1) * (0.5 * np.pi / (nx + 1.0)))
    ty = np.sin(np.arange(1, ny + 1) * (0.5 * np.pi / (ny + 1.0)))
    tz = np.sin(np.arange(1, nz + 1) * (0.5 * np.pi / (nz + 1.0)))
    if nz == 1:
        tz = np.zeros(1)
    ev = 4 * (tx[:, None, None] ** 2 + ty[None, :, None] ** 2 + tz[None, None, :] ** 2)
    ev = ev.ravel()
    slack = EVSL_DBL_EPS_MULT * DBL_EPS
    ev = ev[(ev >= a - slack) & (ev <= b + slack)]
    return np.sort(ev)


def csr_matvec(ia, ja, a, x):
    """y = A x with each row summed left to right (SRC/spmat.c:257-298)."""
    n = len(ia) - 1
    prod = a * x[ja]
    y = np.zeros(n)
    lens = np.diff(ia)
    # Position j of every row is added in turn: the same left-to-right order
    # (r = 0; r += a*x ...) as the reference loop, so results are bitwise equal.
    for j in range(int(lens.max()) if n else 0):
        rows = np.flatnonzero(lens > j)
        y[rows] = y[rows] + prod[ia[rows] + j]
    return y


def _trig(fn, j0, j1, th):
    """fn(j * th) for j = j0 .. j1-1 through the C library's sin / cos (the
    functions the reference calls; numpy's vectorised ones may round the last
    bit differently)."""
    return np.array([fn(j * th) for j in range(j0, j1)], dtype=np.float64)


def _seqsum(t):
    """Left-to-right sum (the reference's loops), not numpy's pairwise sum."""
    return float(np.cumsum(t)[-1]) if len(t) else 0.0


def dampcf(m, damping):
    """Damping coefficients jac[0..m] (SRC/chebpoly.c:39-66)."""
    jac = np.empty(m + 1)
    jac[0] = 0.5
    if m < 1:
        return jac
    k = np.arange(1, m + 1, dtype=np.float64)
    if damping == 0:
        jac[1:] = 1.0
    elif damping == 1:
        thetJ = EVSL_PI / (m + 2.0)
        a1 = 1.0 / (m + 2.0)
        a2 = math.sin(thetJ)
        jac[1:] = a1 * _trig(math.sin, 2, m + 2, thetJ) / a2 + (1 - (k + 1) * a1) * _trig(math.cos, 1, m + 1, thetJ)
    else:
        thetL = EVSL_PI / (m + 1.0)
        jac[1:] = _trig(math.sin, 1, m + 1, thetL) / (k * thetL)
    return jac


def _dif_eval(v, m, thc, jac):
    """sum_j v_j cos(j thc) jac_j, summed left to right (SRC/chebpoly.c:78-84)."""
    return _seqsum(v[:m + 1] * _trig(math.cos, 0, m + 1, thc) * jac[:m + 1])


def _chebx_pltd(m, mu, x):
    """p(x) = sum_k mu_k T_k(x) by the three-term recurrence (SRC/chebpoly.c:105-135)."""
    x = np.atleast_1d(np.asarray(x, dtype=np.float64))
    vkm1 = np.zeros_like(x)
    vk = np.ones_like(x)
    y = np.full_like(x, mu[0])
    for k in range(m):
        scal = 1.0 if k == 0 else 2.0
        vkp1 = scal * x * vk - vkm1
        vkm1, vk = vk, vkp1
        y = y + mu[k + 1] * vk
    return y


def _rootchb(m, v, jac, tha, thb):
    """Newton balancing of the delta-function centre (SRC/chebpoly.c:288-336).

    Returns (ok, mu, thc)."""
    max_iter = 30
    tol_bal = abs(tha - thb) * 1e-13
    thc = 0.5 * (tha + thb)
    fb = _dif_eval(v, m, thb, jac)
    fa = _dif_eval(v, m, tha, jac)
    if fa > 0 or fb < 0:
        return False, None, thc
    j = np.arange(1, m + 1, dtype=np.float64)
    for _ in range(max_iter + 1):
        fval = _dif_eval(v, m, thc, jac)
        d = _seqsum(jac[1:m + 1] * j * _trig(math.sin, 1, m + 1, thc) * v[1:m + 1])
        thN = thc + fval / d
        if abs(fval) < tol_bal or abs(thc - thN) < DBL_EPS * abs(thc):
            break
        if fval > 0:
            if thN < thb or thN > tha:
                thN = 0.5 * (thc + tha)
            thb = thc
            thc = thN
        else:
            if thN < thb or thN > tha:
                thN = 0.5 * (thc + thb)
            tha = thc
            thc = thN
    mu = _trig(math.cos, 0, m + 1, thc) * jac[:m + 1]
    return True, mu, thc


def _chext(max_deg, thresh, deg, aIn, bIn):
    """End-interval filter: scaled Chebyshev polynomial in the Chebyshev basis
    (SRC/chebpoly.c:170-259).  Returns (mu, deg, bar, gam)."""
    if deg > 0:
        thresh = -1.0
        max_deg = deg
    delta = 0.1 * math.sqrt((bIn - aIn) * 0.5)
    eps = 1e-13
    if bIn >= 1.0 - eps:
        x = aIn
        b = x - delta
        a = -1.0
        gam = 1.0
    else:
        x = bIn
        a = x + delta
        b = 1.0
        gam = -1.0
    e = (b - a) * 0.5
    c = (b + a) * 0.5
    sigma1 = e / (gam - c)
    sigma = sigma1
    m1 = max_deg + 1
    t0 = np.zeros(m1)
    t1 = np.zeros(m1)
    t0[0] = 1.0
    t1[0] = -c * (sigma1 / e)
    t1[1] = sigma1 / e
    g0 = 1.0
    g1 = (x - c) * sigma1 / e
    mbest = 0
    if g1 < thresh:
        mbest = 1
    else:
        for k in range(2, max_deg + 1):
            sigma_new = 1.0 / (2.0 / sigma1 - sigma)
            s1 = sigma_new / e
            s2 = 2 * s1 * c
            s3 = sigma * sigma_new
            tnew = np.zeros(m1)
            tnew[1:k] = s1 * (t1[2:k + 1] + t1[0:k - 1])
            tnew[1] = tnew[1] + s1 * t1[0]
            tnew[0] = s1 * t1[1]
            tnew[k] = s1 * t1[k - 1]
            tnew[:k + 1] = tnew[:k + 1] - s2 * t1[:k + 1] - s3 * t0[:k + 1]
            t0 = t1.copy()
            t1 = tnew
            gnew = 2 * (x - c) * s1 * g1 - s3 * g0
            g0 = g1
            g1 = gnew
            mbest = k
            if g1 < thresh:
                break
            sigma = sigma_new
    return t1[:mbest + 1].copy(), mbest, g1, gam


def find_pol(intv, *, damping=2, thresh_int=0.8, thresh_ext=0.2, max_deg=10000, deg=0,
             intvtol=1e-9):
    """Filter design (SRC/chebpoly.c:363-490; defaults SRC/chebpoly.c:15-24).

    Returns a dict with type, deg, mu[0..deg], cc, dd, gam, bar, or None for an
    invalid interval (the reference returns -1)."""
    a, b, lmin, lmax = [float(t) for t in intv]
    if a >= b or a >= lmax or b <= lmin:
        return None
    aa = max(a, lmin)
    bb = min(b, lmax)
    cc = 0.5 * (lmax + lmin)
    dd = 0.5 * (lmax - lmin)
    aa = (aa - cc) / dd
    bb = (bb - cc) / dd
    aa = max(aa, -1.0)
    bb = min(bb, 1.0)
    thb = math.acos(bb)
    tha = math.acos(aa)
    if aa - intvtol <= -1.0:
        ptype, nitv, aa, gam = 1, 1, -1.0, -1.0
    elif bb + intvtol >= 1.0:
        ptype, nitv, bb, gam = 2, 1, 1.0, 1.0
    else:
        ptype, nitv = 0, 2
    if nitv == 1:
        mu, mbest, bar, gam = _chext(max_deg, thresh_ext, deg, aa, bb)
        return dict(type=ptype, deg=mbest, mu=mu, cc=cc, dd=dd, gam=gam, bar=bar)
    min_deg = int(2 + 0.5 / (bb - aa))
    min_deg = max(min_deg, 2)
    min_deg = min(min_deg, (max_deg + 1) // 2)
    thresh = thresh_int
    if deg > 0:
        thresh = -1
        max_deg = deg
    v = np.zeros(max_deg + 1)
    v[:min_deg] = _trig(math.cos, 0, min_deg, thb) - _trig(math.cos, 0, min_deg, tha)
    mu = None
    t = 0.0
    vals = np.array([np.nan, np.nan])
    m = min_deg
    accepted = False
    while m < max_deg:
        jac = dampcf(m, damping)
        v[m] = math.cos(m * thb) - math.cos(m * tha)
        ok, mu_m, thc = _rootchb(m, v, jac, tha, thb)
        if not ok:
            m += 1
            continue
        mu = mu_m
        gam = math.cos(thc)
        t = float(_chebx_pltd(m, mu, gam)[0])
        vals = _chebx_pltd(m, mu, np.array([aa, bb]))
        if vals[0] <= t * thresh and vals[1] <= t * thresh:
            accepted = True
            break
        m += 1
    mbest = m if accepted else m - 1
    mu = mu[:mbest + 1] / t
    return dict(type=0, deg=mbest, mu=mu, cc=cc, dd=dd, gam=gam, bar=min(vals[0], vals[1]) / t)


def cheb_av(pol, ia, ja, a, v):
    """y = p((A - cc)/dd) v by the three-term recurrence (SRC/chebpoly.c:519-598),
    in the reference CPU build's operation order (daxpy, dscal, daxpy, daxpy)."""
    mu, cc, dd, m = pol["mu"], pol["cc"], pol["dd"], pol["deg"]
    vk = v.copy()
    vkm1 = np.zeros_like(v)
    y = mu[0] * v
    for k in range(1, m + 1):
        t = (1.0 / dd) if k == 1 else (2.0 / dd)
        vkp1 = csr_matvec(ia, ja, a, vk)
        vkp1 = vkp1 + (-cc) * vk
        vkp1 = t * vkp1
        if k > 1:
            vkp1 = vkp1 + (-1.0) * vkm1
        y = y + mu[k] * vkp1
        vkm1, vk = vk, vkp1
    return y


def kpmdos(Mdeg, damping, probes, intv, ia, ja, a):
    """KPM DOS moments and eigenvalue count (SRC/spslice.c:29-148), probes given
    explicitly (nvec x n); each is normalised inside as the reference does."""
    lmin, lmax = intv[2], intv[3]
    aa = max(intv[0], lmin)
    bb = min(intv[1], lmax)
    ctr = (lmax + lmin) / 2.0
    wid = (lmax - lmin) / 2.0
    beta1 = math.acos(max(-1.0 + DBL_EPS, (aa - ctr) / wid))
    beta2 = math.acos(min(1.0 - DBL_EPS, (bb - ctr) / wid))
    jac = dampcf(Mdeg, damping)
    jac[0] = 1.0
    mu = np.zeros(Mdeg + 1)
    tcnt = 0.0
    probes = np.atleast_2d(probes)
    n = probes.shape[1]
    for p in probes:
        v = p * (1.0 / np.linalg.norm(p))
        vk = v.copy()
        vkm1 = np.zeros(n)
        mu[0] += jac[0]
        tcnt -= jac[0] * (beta2 - beta1)
        for k in range(Mdeg):
            vkp1 = csr_matvec(ia, ja, a, vk)
            scal = (1.0 if k == 0 else 2.0) / wid
            vkp1 = vkp1 + (-ctr) * vk
            vkp1 = scal * vkp1
            vkp1 = vkp1 + (-1.0) * vkm1
            vkm1, vk = vk, vkp1
            k1 = k + 1
            t = 2 * jac[k1] * float(np.dot(vk, v))
            mu[k1] += t
            tcnt -= t * (math.sin(k1 * beta2) - math.sin(k1 * beta1)) / k1
    t = 1.0 / (probes.shape[0] * np.pi)
    return mu * t, tcnt * t * n


def int_chx(mu, xi):
    """Integrals of the KPM DOS from xi[0] to xi[j] (SRC/spslice.c:155-181)."""
    thetas = np.arccos(xi)
    theta0 = thetas[0]
    yi = mu[0] * (theta0 - thetas)
    for k in range(1, len(mu)):
        yi = yi + mu[k] * (math.sin(k * theta0) / k - np.sin(k * thetas) / k)
    return yi


def linspace(a, b, num):
    """EVSL's linspace with exact end points (SRC/vect.c:82-92)."""
    h = 0.0 if num == 1 else (b - a) / (num - 1)
    arr = a + np.arange(num) * h
    arr[0] = a
    arr[-1] = b
    return arr


def spslicer(mu, intv, n_int, npts):
    """Equal-count slicing from the KPM DOS (SRC/spslice.c:205-297).
    Returns (err, sli)."""
    a, b, lmin, lmax = intv
    if a >= b or a >= lmax or b <= lmin:
        return -1, None
    aa = max(a, lmin)
    bb = min(b, lmax)
    sli = np.zeros(n_int + 1)
    if n_int == 1:
        sli[0], sli[1] = a, b
        return 0, sli
    ctr = (lmax + lmin) / 2
    wid = (lmax - lmin) / 2
    aL = max((aa - ctr) / wid, -1.0)
    bL = min((bb - ctr) / wid, 1.0)
    npts = max(npts, 2 * n_int + 1)
    xi = linspace(aL, bL, npts)
    yi = int_chx(mu, xi)
    target = yi[npts - 1] / n_int
    ls = 0
    ii = 0
    sli[0] = a
    while True:
        ls += 1
        if ls >= n_int:
            break
        while ii < npts and yi[ii] < target:
            ii += 1
        if ii == npts:
            break
        if (target - yi[ii - 1]) < (yi[ii] - target):
            ii -= 1
        sli[ls] = ctr + wid * xi[ii]
        target = yi[ii] + (yi[npts - 1] - yi[ii]) / (n_int - ls)
    sli[n_int] = b
    err = 1 if ls != n_int else 0
    if np.any(sli[1:] < sli[:-1]):
        err += 2
    return err, sli


def cgs_dgks(V, v):
    """Classical Gram-Schmidt with the DGKS stop, at most NGS_MAX passes
    (SRC/misc_la.c:221-261).  Returns (v, norm)."""
    eta = 1.0 / math.sqrt(2.0)
    old = np.linalg.norm(v)
    new = 0.0
    for _ in range(NGS_MAX):
        w = V.T @ v
        v = v - V @ w
        new = np.linalg.norm(v)
        if new > eta * old:
            break
        old = new
    return v, new


def cheblan_nr(intv, maxit, tol, vinit, pol, ia, ja, a, restart_vectors=()):
    """Non-restarted filtered Lanczos (SRC/cheblanNr.c:57-434) for small n.

    Eigenvalues of the tridiagonal matrix use scipy's eigh_tridiagonal in
    place of LAPACK dstev.  Returns (lam, Y (nev x n), res) in the
    reference's output order."""
    from scipy.linalg import eigh_tridiagonal

    n = len(vinit)
    maxit = min(n, maxit)
    bar, gamB = pol["bar"], pol["gam"]
    aa, bb = intv[0], intv[1]
    V = np.zeros((maxit + 1, n))
    dT = np.zeros(maxit)
    eT = np.zeros(maxit)
    restarts = list(restart_vectors)
    V[0] = cheb_av(pol, ia, ja, a, vinit)
    V[0] *= 1.0 / np.linalg.norm(V[0])
    wn, nwn, tr0, beta = 0.0, 0, 0.0, 0.0
    kdim = 0
    k = 0
    while k < maxit:
        v = V[k]
        znew = cheb_av(pol, ia, ja, a, v)
        if k > 0:
            znew = znew + (-beta) * V[k - 1]
        alpha = float(np.dot(v, znew))
        dT[k] = alpha
        wn += abs(alpha)
        znew = znew + (-alpha) * v
        znew, beta = cgs_dgks(V[:k + 1].T, znew)
        wn += 2.0 * beta
        nwn += 3
        if beta * nwn < ORTH_TOL * wn:
            vr = restarts.pop(0)
            znew = cheb_av(pol, ia, ja, a, vr)
            znew, beta = cgs_dgks(V[:k + 1].T, znew)
            znew = znew * (1.0 / beta)
            beta = 0.0
        else:
            znew = znew * (1.0 / beta)
        V[k + 1] = znew
        eT[k] = beta
        if (k < 30 or (k - 30) % 20 != 0) and k != maxit - 1:
            k += 1
            continue
        kdim = k + 1
        ev = eigh_tridiagonal(dT[:kdim], eT[:kdim - 1], eigvals_only=True)
        sel = ev + EVSL_DBL_EPS_MULT * DBL_EPS >= bar
        tr1 = float(np.sum(ev[sel]))
        if abs(tr1 - tr0) < 2e-12 or abs(tr1) + abs(tr0) < 1e-10:
            break
        tr0 = tr1
        k += 1
    ev, Z = eigh_tridiagonal(dT[:kdim], eT[:kdim - 1])
    lam, Y, res = [], [], []
    slack = EVSL_DBL_EPS_MULT * DBL_EPS
    for i in range(kdim):
        if ev[i] < bar:
            continue
        u = V[:kdim].T @ Z[:, i]
        u = u * (1.0 / np.linalg.norm(u))
        w = csr_matvec(ia, ja, a, u)
        t = float(np.dot(w, u))
        if t < aa - slack or t > bb + slack:
            continue
        r = float(np.linalg.norm(w - t * u))
        if r < tol:
            lam.append(t)
            Y.append(u)
            res.append(r)
    return np.array(lam), np.array(Y).reshape(len(lam), n), np.array(res), kdim


def lan_bounds(msteps, v, ia, ja, a):
    """Spectrum bounds from a short Lanczos run with one modified Gram-Schmidt
    reorthogonalisation pass per step (SRC/lanbounds.c:21-129, standard
    problem).  On a lucky breakdown the reference keeps the squared beta as
    the bottom coupling; so does this.  Tridiagonal eigenpairs use scipy's
    eigh_tridiagonal in place of SymmTridEig."""
    from scipy.linalg import eigh_tridiagonal

    n = len(v)
    msteps = min(n, msteps)
    V = np.zeros((msteps + 1, n))
    alp = np.zeros(msteps)
    bet = np.zeros(msteps)
    V[0] = v * (1.0 / np.linalg.norm(v))
    wn = 0.0
    for j in range(msteps):
        z = csr_matvec(ia, ja, a, V[j])
        if j:
            z = z + (-bet[j - 1]) * V[j - 1]
        alp[j] = z @ V[j]
        wn += alp[j] * alp[j]
        z = z + (-alp[j]) * V[j]
        for i in range(j + 1):
            z = z + (-(z @ V[i])) * V[i]
        V[j + 1] = z
        bet[j] = z @ z
        if bet[j] * (j + 1) < ORTH_TOL * wn:
            msteps = j + 1
            break
        wn += 2.0 * bet[j]
        bet[j] = math.sqrt(bet[j])
        V[j + 1] *= 1.0 / bet[j]
    bottom = bet[msteps - 1]
    w, S = eigh_tridiagonal(alp[:msteps], bet[:msteps - 1])
    return w[0] - abs(bottom * S[msteps - 1, 0]), w[-1] + abs(bottom * S[msteps - 1, msteps - 1])


def _orth(V):
    """Column orthonormalisation (SRC/misc_la.c:317-341): rows of V are the
    columns; each one CGS-DGKS'd against the previous and normalised."""
    out = np.array(V, dtype=np.float64, copy=True)
    out[0] *= 1.0 / np.linalg.norm(out[0])
    for i in range(1, len(out)):
        w, nrm = cgs_dgks(out[:i].T, out[i])
        out[i] = w * (1.0 / nrm)
    return out


def cheb_si(nev, intv, maxit, tol, vinit_block, pol, ia, ja, a):
    """Polynomial-filtered subspace iteration (SRC/chebsi.c:39-335) for small
    n: V <- orth(p(A) V) with the active block kept orthogonal to the locked
    one; every 5 iterations a Rayleigh-Ritz step with p(A), candidates with
    p(A)-residual < tol/100 confirmed by the A-residual < tol and locked; stop
    when every column is locked or 2 locked values lie outside [a, b].
    Rows of vinit_block are the start columns.  Returns (lam, Y, res) of the
    locked pairs inside [a, b], in locking order."""
    NBUF, CVCHECK = 2, 5
    tolP = tol * 0.01
    aa, bb = intv[0], intv[1]
    lo_ok, hi_ok = aa - EVSL_DBL_EPS_MULT * DBL_EPS, bb + EVSL_DBL_EPS_MULT * DBL_EPS
    V = _orth(vinit_block)
    PV = np.array([cheb_av(pol, ia, ja, a, x) for x in V])
    Lam, res = np.zeros(nev), np.zeros(nev)
    nlock, nact, nlock_ab, it, find_more = 0, nev, 0, 0, True
    while it < maxit and find_more:
        V[nlock:] = PV[nlock:]
        if nlock:
            V[nlock:] -= (V[nlock:] @ V[:nlock].T) @ V[:nlock]
        V[nlock:] = _orth(V[nlock:])
        PV[nlock:] = np.array([cheb_av(pol, ia, ja, a, x) for x in V[nlock:]])
        if nlock:
            PV[nlock:] -= (PV[nlock:] @ V[:nlock].T) @ V[:nlock]
        if (it + 1) % CVCHECK == 0 or it + 1 == maxit:
            T = V[nlock:] @ PV[nlock:].T
            evalT, evecT = np.linalg.eigh(0.5 * (T + T.T))
            V[nlock:] = evecT.T @ V[nlock:]
            PV[nlock:] = evecT.T @ PV[nlock:]
            locked, active = [], []
            for i in range(nlock, nev):
                r = PV[i] - evalT[i - nlock] * V[i]
                if np.linalg.norm(r) < tolP:
                    Av = csr_matvec(ia, ja, a, V[i])
                    rq = V[i] @ Av
                    ra = np.linalg.norm(Av - rq * V[i])
                    if ra < tol:
                        Lam[nlock + len(locked)] = rq
                        res[nlock + len(locked)] = ra
                        locked.append(i)
                        continue
                active.append(i)
            order = locked + active
            V[nlock:] = V[order]
            PV[nlock:] = PV[order]
            nlock_ab += sum(1 for k in range(len(locked)) if lo_ok <= Lam[nlock + k] <= hi_ok)
            nlock += len(locked)
            nact = len(active)
            if nlock - nlock_ab >= NBUF or nlock == nev:
                find_more = False
        it += 1
    keep = [i for i in range(nlock) if lo_ok <= Lam[i] <= hi_ok]
    return Lam[keep], V[keep], res[keep]


def read_coo_mm(path, idxin=1, idxout=0):
    """Matrix-Market coordinate reader (TESTS/COMMON/io.c:115-214 with the
    banner/size rules of TESTS/COMMON/mmio.c:80-210).  Returns (rc, n, ir,
    jc, vv); rc 1 for an unsupported or malformed header, -1 for a short
    file.  Symmetric files: the transposed off-diagonal entries are appended
    after the stored ones, in file order."""
    with open(path, "r") as f:
        lines = f.read().split("\n")
    tok = lines[0].split()
    if len(tok) < 5 or not tok[0].startswith("%%MatrixMarket"):
        return 1, 0, None, None, None
    obj, fmt, field, sym = (t.lower() for t in tok[1:5])
    if obj != "matrix" or fmt != "coordinate" or field not in ("real", "integer") or \
            sym not in ("general", "symmetric", "skew-symmetric"):
        return 1, 0, None, None, None
    k = 1
    while k < len(lines) and lines[k].startswith("%"):
        k += 1
    rest = " ".join(lines[k:]).split()
    if len(rest) < 3:
        return 1, 0, None, None, None
    nrow, ncol, nnz = int(rest[0]), int(rest[1]), int(rest[2])
    if nrow != ncol:
        return 1, 0, None, None, None
    vals = rest[3:3 + 3 * nnz]
    if len(vals) < 3 * nnz:
        return -1, 0, None, None, None
    ir = np.array([int(float(t)) for t in vals[0::3]], dtype=np.int32)
    jc = np.array([int(float(t)) for t in vals[1::3]], dtype=np.int32)
    vv = np.array([float(t) for t in vals[2::3]])
    if sym == "symmetric":
        off = ir != jc
        ir, jc, vv = (np.concatenate([ir, jc[off]]), np.concatenate([jc, ir[off]]), np.concatenate([vv, vv[off]]))
    off = idxout - idxin
    return 0, nrow, ir + off, jc + off, vv


def coo_to_csr(n, ir, jc, vv, cooidx=0):
    """cooMat_to_csrMat + sortrow (SRC/spmat.c:160-190, :67-85): rows in
    order, each row stably sorted by column (ties in input order)."""
    r = np.asarray(ir, dtype=np.int64) - cooidx
    c = np.asarray(jc, dtype=np.int64) - cooidx
    order = np.lexsort((np.arange(len(r)), c, r))
    ia = np.zeros(n + 1, dtype=np.int64)
    np.add.at(ia, r + 1, 1)
    return np.cumsum(ia).astype(np.int32), c[order].astype(np.int32), np.asarray(vv, dtype=np.float64)[order]


def simpson(xi, yi):
    """Cumulative Simpson integral (SRC/simpson.c:25-50), returned as a new
    array."""
    y = np.array(yi, dtype=np.float64)
    npts = len(y)
    tc = 0.0
    i = 1
    ysav = y[0]
    y[0] = 0.0
    while i < npts - 1:
        ti = (xi[i] - xi[i - 1]) * (ysav + y[i]) / 2.0
        tm = tc + ti
        ti = (xi[i + 1] - xi[i - 1]) * (ysav + 4 * y[i] + y[i + 1]) / 6.0
        tc += ti
        y[i] = tm
        ysav = y[i + 1]
        y[i + 1] = tc
        i += 2
    if i == npts - 1:
        ti = (xi[i] - xi[i - 1]) * (y[i] + ysav) / 2.0
        y[i] = tc + ti
    return y


def spslicer2(xi, yi, n_int):
    """Equal-count slices from a DOS curve (SRC/spslice2.c:25-45)."""
    y = simpson(xi, yi)
    npts = len(y)
    t = y[0]
    want = (y[npts - 1] - y[0]) / float(n_int)
    sli = np.zeros(n_int + 1)
    sli[0] = xi[0]
    ls = 0
    for k in range(1, npts):
        if y[k] - t >= want:
            ls += 1
            if ls <= n_int:
                sli[ls] = xi[k]
            t = y[k]
    sli[n_int] = xi[npts - 1]
    return sli


def _dos_params(msteps_or_n, intv):
    lm, lM = intv[2], intv[3]
    M = min(msteps_or_n, 30)
    H = (lM - lm) / (M - 1)
    sigma = H / math.sqrt(8 * math.log(1.25))
    sigma2 = 2 * sigma * sigma
    width = sigma * math.sqrt(-2.0 * math.log(1e-08))
    return sigma2, width


def exdos(vals, npts, intv):
    """DOS of known eigenvalues (SRC/exDOS.c:17-67): (rc, x, y)."""
    n = len(vals)
    sigma2, width = _dos_params(n, intv)
    a, b = intv[0], intv[1]
    x = linspace(a, b, npts)
    h = x[1] - x[0]
    y = np.zeros(npts)
    j = 0
    for t in vals:
        if t < a or t > b:
            continue
        j = max(int((t - a - width) / h), 0)
        xi = a + j * h
        while xi <= min(t + width, b) and j < npts:
            y[j] += math.exp(-(xi - t) * (xi - t) / sigma2)
            j += 1
            xi += h
    if j == 0:
        return 1, x, y
    scaling = 1.0 / (n * math.sqrt(sigma2 * math.pi))
    return 0, x, scaling * y


def library_normal(seed, draw, n):
    """randn_double_device of the GPU library and the oracle hook: Box-Muller
    on the uniform draws 2i and 2i+1 of draw d."""
    u = library_uniform(seed, draw, 2 * n)
    u1 = np.maximum(0.5 * (u[0::2] + 1.0), 1e-300)
    u2 = 0.5 * (u[1::2] + 1.0)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


def lan_dos(nvec, msteps, npts, intv, ia, ja, a, seed):
    """Lanczos DOS (SRC/landos.c:37-200) for small n with the library's
    normal draws (one per vector, starting at draw 0 after seeding).  One
    modified Gram-Schmidt pass per step as in the reference; tridiagonal
    eigenpairs from scipy.  Returns (x, y, neig)."""
    from scipy.linalg import eigh_tridiagonal

    n = len(ia) - 1
    lm, lM = intv[2], intv[3]
    tol_bd = 1.e-13 * (abs(lM) + abs(lm))
    aa, bb = max(intv[0], intv[2]), min(intv[1], intv[3])
    sigma2, width = _dos_params(msteps, intv)
    x = linspace(aa, bb, npts)
    y = np.zeros(npts)
    draw = 0
    for _ in range(nvec):
        v = library_normal(seed, draw, n)
        draw += 1
        V = np.zeros((msteps + 1, n))
        V[0] = v * (1.0 / math.sqrt(v @ v))
        alp, bet = np.zeros(msteps), np.zeros(msteps)
        wn = 0.0
        for j in range(msteps):
            z = csr_matvec(ia, ja, a, V[j])
            if j:
                z = z + (-bet[j - 1]) * V[j - 1]
            alp[j] = z @ V[j]
            wn += alp[j] * alp[j]
            z = z + (-alp[j]) * V[j]
            for i in range(j + 1):
                z = z + (-(z @ V[i])) * V[i]
            bet[j] = z @ z
            if bet[j] * (j + 1) < ORTH_TOL * wn:
                msteps = j + 1
                break
            if bet[j] > tol_bd:
                wn += 2.0 * bet[j]
                bet[j] = math.sqrt(bet[j])
                V[j + 1] = z * (1.0 / bet[j])
            else:
                draw += 1
                for i in range(j + 1):
                    z = z + (-(z @ V[i])) * V[i]
                bet[j] = z @ z
                wn += 2.0 * bet[j]
                V[j + 1] = z * (1.0 / math.sqrt(bet[j]))
                bet[j] = 0.0
        w, S = eigh_tridiagonal(alp[:msteps], bet[:msteps - 1])
        g2 = S[0, :] ** 2
        for i in range(msteps):
            near = np.abs(x - w[i]) < width
            y[near] += g2[i] * np.exp(-((x[near] - w[i]) * (x[near] - w[i])) / sigma2)
    y = (1.0 / (nvec * math.sqrt(sigma2 * math.pi))) * y
    integ = simpson(x, y)
    return x, y, integ[-1] * n


# ---------------------------------------------------------------------------
# Seeded inputs shared by tests and bench
# ---------------------------------------------------------------------------

def seeded_normal(n, seed):
    """Standard-normal start vector, normalised (the workloads' vinit)."""
    v = np.random.default_rng(seed).standard_normal(n)
    return v / np.linalg.norm(v)


def seeded_rademacher(nvec, n, seed):
    """Rademacher (+-1) KPM probes."""
    return np.random.default_rng(seed).choice(np.array([-1.0, 1.0]), size=(nvec, n))


def _mix64(z):
    """SplitMix64 output function on uint64 numpy arrays."""
    z = (z + np.uint64(0x9E3779B97F4A7C15)).astype(np.uint64)
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)).astype(np.uint64)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)).astype(np.uint64)
    return z ^ (z >> np.uint64(31))


def library_uniform(seed, draw, n):
    """The counter-based generator behind rand_double_device of both the GPU
    library and the oracle hook (oracle/ref_hooks.c): value i of draw d is
    mix64(seed*0x9E3779B97F4A7C15 + (d << 32) + i) mapped to [-1, 1)."""
    with np.errstate(over="ignore"):
        key = (np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15) + (np.uint64(draw) << np.uint64(32))
               + np.arange(n, dtype=np.uint64))
        u = (_mix64(key) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return 2.0 * u - 1.0


def kpm_raw_dots(Mdeg, probes, intv, ia, ja, a):
    """Raw KPM products dots[k, m] = (T_{k+1}(A~) v_m) . v_m of the normalised
    probes (the quantities kpmdos accumulates, SRC/spslice.c:101-125)."""
    lmin, lmax = intv[2], intv[3]
    ctr = (lmax + lmin) / 2.0
    wid = (lmax - lmin) / 2.0
    probes = np.atleast_2d(probes)
    out = np.zeros((Mdeg, probes.shape[0]))
    for m, p in enumerate(probes):
        v = p * (1.0 / np.linalg.norm(p))
        vk = v.copy()
        vkm1 = np.zeros_like(v)
        for k in range(Mdeg):
            vkp1 = csr_matvec(ia, ja, a, vk)
            scal = (1.0 if k == 0 else 2.0) / wid
            vkp1 = vkp1 + (-ctr) * vk
            vkp1 = scal * vkp1
            vkp1 = vkp1 + (-1.0) * vkm1
            vkm1, vk = vk, vkp1
            out[k, m] = float(np.dot(vk, v))
    return out


def kpm_raw_dots_exact(Mdeg, probes, intv, ia, ja, a):
    """kpm_raw_dots with each dot product (T_{k+1}(A~) v_m) . v_m of the
    reference's FP64 vectors accumulated in extended precision (numpy
    longdouble: 64-bit significand products and sums) and rounded once: the
    dots of the reference's own recurrence without the rounding error of a
    sequential FP64 sum over n terms (SRC/spslice.c:101-125 forms them with
    one FP64 ddot per degree)."""
    lmin, lmax = intv[2], intv[3]
    ctr = (lmax + lmin) / 2.0
    wid = (lmax - lmin) / 2.0
    probes = np.atleast_2d(probes)
    out = np.zeros((Mdeg, probes.shape[0]))
    for m, p in enumerate(probes):
        v = p * (1.0 / np.linalg.norm(p))
        vl = v.astype(np.longdouble)
        vk = v.copy()
        vkm1 = np.zeros_like(v)
        for k in range(Mdeg):
            vkp1 = csr_matvec(ia, ja, a, vk)
            scal = (1.0 if k == 0 else 2.0) / wid
            vkp1 = vkp1 + (-ctr) * vk
            vkp1 = scal * vkp1
            vkp1 = vkp1 + (-1.0) * vkm1
            vkm1, vk = vk, vkp1
            out[k, m] = float(np.sum(vk.astype(np.longdouble) * vl))
    return out


def kpm_moments_from_dots(Mdeg, damping, n, intv, dots):
    """The accumulation of kpmdos (SRC/spslice.c:101-148) from raw dots
    (Mdeg x nvec), in the reference's probe-major order."""
    lmin, lmax = intv[2], intv[3]
    aa = max(intv[0], lmin)
    bb = min(intv[1], lmax)
    ctr = (lmax + lmin) / 2.0
    wid = (lmax - lmin) / 2.0
    beta1 = math.acos(max(-1.0 + DBL_EPS, (aa - ctr) / wid))
    beta2 = math.acos(min(1.0 - DBL_EPS, (bb - ctr) / wid))
    jac = dampcf(Mdeg, damping)
    jac[0] = 1.0
    mu = np.zeros(Mdeg + 1)
    tcnt = 0.0
    nvec = dots.shape[1]
    for m in range(nvec):
        mu[0] += jac[0]
        tcnt -= jac[0] * (beta2 - beta1)
        for k in range(Mdeg):
            k1 = k + 1
            t = 2 * jac[k1] * float(dots[k, m])
            mu[k1] += t
            tcnt -= t * (math.sin(k1 * beta2) - math.sin(k1 * beta1)) / k1
    t = 1.0 / (nvec * np.pi)
    return mu * t, tcnt * t * n


def kpm_raw_dots_identities(Mdeg, probes, intv, ia, ja, a):
    """The same raw KPM products through the Chebyshev product identities
    (T_2k = 2 T_k^2 - T_0, T_2k+1 = 2 T_k+1 T_k - T_1): with w_j = T_j(A~) v,
    mu_2k+2 = 2 <w_k+1, w_k+1> - <w_0, w_0> and mu_2k+1 = 2 <w_k+1, w_k> - mu_1
    (mu_1 = <w_1, w_0>), from ceil(Mdeg/2) products -- the restatement of the
    library's two-moments-per-step KPM, checked against kpm_raw_dots."""
    lmin, lmax = intv[2], intv[3]
    ctr = (lmax + lmin) / 2.0
    wid = (lmax - lmin) / 2.0
    probes = np.atleast_2d(probes)
    K = (Mdeg + 1) // 2
    out = np.zeros((Mdeg, probes.shape[0]))
    for m, p in enumerate(probes):
        v = p * (1.0 / np.linalg.norm(p))
        c0 = float(np.dot(v, v))
        wk, wkm1 = v.copy(), np.zeros_like(v)
        mu1 = 0.0
        for k in range(K):
            scal = (1.0 if k == 0 else 2.0) / wid
            w = scal * (csr_matvec(ia, ja, a, wk) + (-ctr) * wk) - wkm1
            a_k, b_k = float(np.dot(w, w)), float(np.dot(w, wk))
            if k == 0:
                mu1 = b_k
            out[2 * k, m] = mu1 if k == 0 else 2.0 * b_k - mu1
            if 2 * k + 1 < Mdeg:
                out[2 * k + 1, m] = 2.0 * a_k - c0
            wkm1, wk = wk, w
    return out
