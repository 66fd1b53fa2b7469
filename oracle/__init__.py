"""ctypes bindings for the FP64 CPU oracle (``libscft_oracle.so``).

TEST INFRASTRUCTURE ONLY.  The oracle restates the reference field solver
(PolymerTheory/SCFT_string: scft.cu, density.h, GPU_kernels.h) in plain C and
is used by ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of
``bench.py`` as the checker.  The product (``scft_string_b200``) never imports
this package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libscft_oracle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class _Problem(C.Structure):
    _fields_ = [
        ("m", C.c_int * 3),
        ("D", C.c_double * 3),
        ("N", C.c_int),
        ("alpha", C.c_double),
        ("ens", C.c_int),
        ("phidb", C.c_double),
        ("chi", C.c_double),
        ("f", C.c_double),
        ("strn", C.c_int),
        ("fix", C.c_int * 2),
        ("dostring", C.c_int),
        ("springsteps", C.c_int),
    ]


class IterRecord(C.Structure):
    _fields_ = [
        ("k", C.c_int),
        ("lam", C.c_double),
        ("errtot", C.c_double),
        ("fitup", C.c_double),
        ("stepav", C.c_double),
        ("did_freee", C.c_int),
        ("FE", C.c_double),
    ]


def build() -> None:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.oc_grid_create.restype = C.c_void_p
        L.oc_grid_create.argtypes = [_ip, _dp]
        L.oc_grid_destroy.argtypes = [C.c_void_p]
        L.oc_fft1d.argtypes = [C.c_int, _dp, C.c_int]
        L.oc_fft_r2c.argtypes = [C.c_void_p, _dp, _dp]
        L.oc_fft_c2r.argtypes = [C.c_void_p, _dp, _dp]
        L.oc_ksq.argtypes = [C.c_void_p, _dp]
        L.oc_density_create.restype = C.c_void_p
        L.oc_density_create.argtypes = [_ip, _dp, C.c_int]
        L.oc_density_destroy.argtypes = [C.c_void_p]
        L.oc_prepare_factors.argtypes = [C.c_void_p, C.c_double, _dp]
        L.oc_do_step.argtypes = [C.c_void_p, _dp, _dp, C.c_int, C.c_int, C.c_int]
        L.oc_props.restype = C.c_int
        L.oc_props.argtypes = [C.c_void_p, _dp, _dp, C.c_int, C.c_double, C.c_double, _dp,
                               C.c_double, C.c_int]
        L.oc_props_fcont.restype = C.c_int
        L.oc_props_fcont.argtypes = L.oc_props.argtypes
        L.oc_stress.restype = C.c_int
        L.oc_stress.argtypes = [C.c_void_p, _dp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, _dp]
        L.oc_stress_fcont.restype = C.c_int
        L.oc_stress_fcont.argtypes = L.oc_stress.argtypes
        L.oc_dlnq_df.restype = C.c_int
        L.oc_dlnq_df.argtypes = L.oc_stress.argtypes
        L.oc_density_q.restype = _dp
        L.oc_density_q.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.oc_density_Q.argtypes = [C.c_void_p, _dp, _dp]
        L.oc_reduction_sum.restype = C.c_double
        L.oc_reduction_sum.argtypes = [_dp, C.c_int]
        L.oc_spline_coeffs.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.oc_spline_derivs.argtypes = [C.c_int, _dp, C.POINTER(_dp), C.c_int, C.c_int, _ip,
                                       C.POINTER(_dp)]
        L.oc_spline_redist.argtypes = [C.c_int, _dp, _dp, C.POINTER(_dp), C.c_int, C.c_int,
                                       _ip, C.c_double]
        L.oc_solver_create.restype = C.c_void_p
        L.oc_solver_create.argtypes = [C.POINTER(_Problem)]
        L.oc_solver_destroy.argtypes = [C.c_void_p]
        L.oc_solver_W.restype = _dp
        L.oc_solver_W.argtypes = [C.c_void_p, C.c_int]
        L.oc_solver_doiis.restype = _ip
        L.oc_solver_doiis.argtypes = [C.c_void_p]
        L.oc_solve_field0.restype = C.c_int
        L.oc_solve_field0.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double]
        L.oc_solve_field.restype = C.c_int
        L.oc_solve_field.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double,
                                     C.POINTER(IterRecord), _dp, _dp]
        L.oc_free_energy.restype = C.c_double
        L.oc_free_energy.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.oc_solver_props_calls.restype = C.c_long
        L.oc_solver_props_calls.argtypes = [C.c_void_p]
        L.oc_edist.restype = C.c_double
        L.oc_edist.argtypes = [_dp, _dp, C.c_int]
        L.oc_set_threads.argtypes = [C.c_int]
        L.oc_get_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def set_threads(n: int) -> None:
    lib().oc_set_threads(int(n))


def get_threads() -> int:
    return lib().oc_get_threads()


def fft1d(x: np.ndarray, sign: int = -1) -> np.ndarray:
    """Complex FFT of a 1-D array (unnormalised; sign -1 forward)."""
    buf = np.ascontiguousarray(np.asarray(x, np.complex128)).view(np.float64).copy()
    n = buf.size // 2
    if lib().oc_fft1d(n, _p(buf), sign) != 0:
        raise ValueError(f"unsupported length {n}")
    return buf.view(np.complex128)


class Grid:
    def __init__(self, m, D):
        self.m = tuple(int(v) for v in m)
        self.D = tuple(float(v) for v in D)
        mi = (C.c_int * 3)(*self.m)
        Di = (C.c_double * 3)(*self.D)
        self.h = lib().oc_grid_create(mi, Di)
        if not self.h:
            raise ValueError("unsupported grid")
        self.M = self.m[0] * self.m[1] * self.m[2]
        self.mk2 = self.m[2] // 2 + 1
        self.Mk = self.m[0] * self.m[1] * self.mk2

    def __del__(self):
        if getattr(self, "h", None):
            lib().oc_grid_destroy(self.h)
            self.h = None

    def r2c(self, a: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(a, np.float64).reshape(-1)
        out = np.zeros(2 * self.Mk)
        lib().oc_fft_r2c(self.h, _p(a), _p(out))
        return out.view(np.complex128).reshape(self.m[0], self.m[1], self.mk2)

    def c2r(self, h: np.ndarray) -> np.ndarray:
        hb = np.ascontiguousarray(h, np.complex128).reshape(-1).view(np.float64).copy()
        out = np.zeros(self.M)
        lib().oc_fft_c2r(self.h, _p(hb), _p(out))
        return out.reshape(self.m)

    def ksq(self) -> np.ndarray:
        out = np.zeros(self.Mk)
        lib().oc_ksq(self.h, _p(out))
        return out.reshape(self.m[0], self.m[1], self.mk2)


class Density:
    """density(Ns, D) of density.h:272 with props / do_step."""

    def __init__(self, m, D, Ns):
        mi = (C.c_int * 3)(*[int(v) for v in m])
        Di = (C.c_double * 3)(*[float(v) for v in D])
        self.h = lib().oc_density_create(mi, Di, int(Ns))
        if not self.h:
            raise ValueError("unsupported grid")
        self.m = tuple(int(v) for v in m)
        self.M = self.m[0] * self.m[1] * self.m[2]
        self.Ns = int(Ns)

    def __del__(self):
        if getattr(self, "h", None):
            lib().oc_density_destroy(self.h)
            self.h = None

    def props(self, w: np.ndarray, Ns, alpha, phic, f, ens):
        """w: 6*M doubles (in [W-, W+], out [phiA, phiB, phih, phicB]).  Returns (lnQ, phis)."""
        assert w.size >= 6 * self.M
        lnQ = C.c_double(0)
        phis = np.zeros(6)
        rc = lib().oc_props(self.h, _p(w), C.byref(lnQ), int(Ns), float(alpha), float(phic),
                            _p(phis), float(f), int(ens))
        if rc != 0:
            raise ValueError("bad props arguments")
        return lnQ.value, phis[:5].copy()

    def props_fcont(self, w: np.ndarray, Ns, alpha, phic, f, ens):
        """The continuous-f variant (f unrounded, junction step n1 = floor(Ns f))."""
        assert w.size >= 6 * self.M
        lnQ = C.c_double(0)
        phis = np.zeros(6)
        rc = lib().oc_props_fcont(self.h, _p(w), C.byref(lnQ), int(Ns), float(alpha), float(phic),
                                  _p(phis), float(f), int(ens))
        if rc != 0:
            raise ValueError("bad props arguments")
        return lnQ.value, phis[:5].copy()

    def stress(self, W2M, Ns, alpha, phic, f, ens, fcont=False):
        """d lnQ / d L_i (3 values) at the fields W2M = [W-, W+]; fcont selects
        the continuous-f chain of props_fcont."""
        out = np.zeros(3)
        fn = lib().oc_stress_fcont if fcont else lib().oc_stress
        rc = fn(self.h, _p(np.ascontiguousarray(W2M, np.float64)), int(Ns), float(alpha),
                float(phic), float(f), int(ens), _p(out))
        if rc != 0:
            raise ValueError("bad stress arguments")
        return out

    def dlnq_df(self, W2M, Ns, alpha, phic, f, ens):
        """d lnQ / df of the continuous-f variant at the fields W2M = [W-, W+]."""
        out = np.zeros(1)
        rc = lib().oc_dlnq_df(self.h, _p(np.ascontiguousarray(W2M, np.float64)), int(Ns), float(alpha),
                              float(phic), float(f), int(ens), _p(out))
        if rc != 0:
            raise ValueError("bad dlnq_df arguments")
        return float(out[0])

    def prepare(self, ds, W2M):
        lib().oc_prepare_factors(self.h, float(ds), _p(np.ascontiguousarray(W2M, np.float64)))

    def do_step(self, qin: np.ndarray, s, n1, n2) -> np.ndarray:
        qin = np.ascontiguousarray(qin, np.float64).reshape(-1)
        out = np.zeros(2 * self.M)
        lib().oc_do_step(self.h, _p(qin), _p(out), int(s), int(n1), int(n2))
        return out

    def q(self, which, s) -> np.ndarray:
        ptr = lib().oc_density_q(self.h, int(which), int(s))
        return np.ctypeslib.as_array(ptr, shape=(self.M,)).copy()

    def Q(self):
        a, b = C.c_double(0), C.c_double(0)
        lib().oc_density_Q(self.h, C.byref(a), C.byref(b))
        return a.value, b.value


def reduction_sum(a: np.ndarray) -> float:
    a = np.ascontiguousarray(a, np.float64)
    return lib().oc_reduction_sum(_p(a), a.size)


def spline_coeffs(x, a):
    x = np.ascontiguousarray(x, np.float64)
    a = np.ascontiguousarray(a, np.float64)
    n = x.size
    c, b, d = np.zeros(n), np.zeros(n), np.zeros(n)
    lib().oc_spline_coeffs(n, _p(x), _p(a), _p(c), _p(b), _p(d))
    return c, b, d


def _ptrs(rows):
    arr = (_dp * len(rows))()
    for i, r in enumerate(rows):
        arr[i] = _p(r)
    return arr


def spline_derivs(x, Wm: np.ndarray, doiis) -> np.ndarray:
    """Wm: (strn, M) W- of every replica.  Returns dW-/dalpha at the knots
    (rows of replicas with doiis != 1 are zero)."""
    strn, M = Wm.shape
    Wm = np.ascontiguousarray(Wm, np.float64)
    out = np.zeros((strn, M))
    rows_in = [Wm[i] for i in range(strn)]
    rows_out = [out[i] for i in range(strn)]
    d = np.ascontiguousarray(doiis, np.int32)
    lib().oc_spline_derivs(strn, _p(np.ascontiguousarray(x, np.float64)), _ptrs(rows_in), 0, M,
                           d.ctypes.data_as(_ip), _ptrs(rows_out))
    return out


def spline_redist(x, xref, Wm: np.ndarray, doiis, lam) -> np.ndarray:
    strn, M = Wm.shape
    Wm = np.ascontiguousarray(Wm, np.float64).copy()
    rows = [Wm[i] for i in range(strn)]
    d = np.ascontiguousarray(doiis, np.int32)
    lib().oc_spline_redist(strn, _p(np.ascontiguousarray(x, np.float64)),
                           _p(np.ascontiguousarray(xref, np.float64)), _ptrs(rows), 0, M,
                           d.ctypes.data_as(_ip), float(lam))
    return Wm


class Solver:
    """The reference's single-process solver state (scft.cu:1029-1051) with
    solve_field0 / solve_field / FreeE."""

    def __init__(self, m, D, N, alpha, ens, phidb, chi, f, strn, fix=(0, 0), dostring=1,
                 springsteps=0):
        p = _Problem()
        p.m = (C.c_int * 3)(*[int(v) for v in m])
        p.D = (C.c_double * 3)(*[float(v) for v in D])
        p.N, p.alpha, p.ens, p.phidb, p.chi = int(N), float(alpha), int(ens), float(phidb), float(chi)
        p.f = float(round(N * f)) / N  # scft.cu:1008
        p.strn = int(strn)
        p.fix = (C.c_int * 2)(*[int(v) for v in fix])
        p.dostring, p.springsteps = int(dostring), int(springsteps)
        self.p = p
        self.h = lib().oc_solver_create(C.byref(p))
        if not self.h:
            raise ValueError("bad problem")
        self.M = int(np.prod(m))
        self.strn = int(strn)

    def __del__(self):
        if getattr(self, "h", None):
            lib().oc_solver_destroy(self.h)
            self.h = None

    def W(self, ii) -> np.ndarray:
        """Live view of replica ii's 7*M array."""
        ptr = lib().oc_solver_W(self.h, int(ii))
        return np.ctypeslib.as_array(ptr, shape=(7 * self.M,))

    def set_fields(self, ii, wm, wp):
        W = self.W(ii)
        W[: self.M] = np.asarray(wm, np.float64).reshape(-1)
        W[self.M: 2 * self.M] = np.asarray(wp, np.float64).reshape(-1)

    def doiis(self) -> np.ndarray:
        ptr = lib().oc_solver_doiis(self.h)
        return np.ctypeslib.as_array(ptr, shape=(self.strn,))

    def solve_field0(self, ii, maxIter, errTol) -> int:
        return lib().oc_solve_field0(self.h, int(ii), int(maxIter), float(errTol))

    def solve_field(self, maxIter, errTol=1e-3, doii=-1):
        rec = (IterRecord * max(1, maxIter))()
        errs = np.zeros(max(1, maxIter) * self.strn)
        errs3 = np.zeros(max(1, maxIter) * self.strn)
        k = lib().oc_solve_field(self.h, int(doii), int(maxIter), float(errTol), rec, _p(errs),
                                 _p(errs3))
        recs = [dict(k=r.k, lam=r.lam, errtot=r.errtot, fitup=r.fitup, stepav=r.stepav,
                     did_freee=r.did_freee, FE=r.FE) for r in rec[:k]]
        return k, recs, errs[: k * self.strn].reshape(k, self.strn), \
            errs3[: k * self.strn].reshape(k, self.strn)

    def free_energy(self):
        s = self.strn
        alf, F0, F1, F, ph = (np.zeros(s) for _ in range(5))
        FE = lib().oc_free_energy(self.h, _p(alf), _p(F0), _p(F1), _p(F), _p(ph))
        return dict(FE=FE, alf=alf, FEs0=F0, FEs1=F1, FEs=F, phctot=ph)

    def props_calls(self) -> int:
        return lib().oc_solver_props_calls(self.h)
