"""scft_string_b200 -- B200 (sm_100a) field solver for SCFT_string.

Python mirror of the reference's solver interface over the C ABI in
``include/scft_b200.h`` (the product is the CUDA library
``libscft_b200.so``; this module only binds it):

* :class:`Density` -- ``density(Ns, D)`` with ``props`` (density.h:272, 344)
* :class:`StringSolver` -- the single-process solver state with
  ``solve_field0`` / ``solve_field`` / ``free_energy`` (scft.cu:516-853)

Importing this module never falls back to a CPU path: if the shared library
is missing or no sm_100a device is present, calls raise :class:`ScftError`.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libscft_b200.so")

SCFT_FP64, SCFT_FP32 = 0, 1
STATUS = {0: "ok", 1: "CUDA error", 2: "NaN detected", 3: "bad input", 4: "timeout",
          5: "out of memory", 6: "unsupported device"}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class ScftError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {msg}")


class Problem(C.Structure):
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
        ("precision", C.c_int),
        ("batched", C.c_int),
        ("device", C.c_int),
        ("fcont", C.c_int),
        ("nostore", C.c_int),
        ("ckpt_K", C.c_int),
    ]


class IterReport(C.Structure):
    _fields_ = [("k", C.c_int), ("lam", C.c_double), ("errtot", C.c_double),
                ("fitup", C.c_double), ("stepav", C.c_double), ("did_freee", C.c_int),
                ("FE", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("props_calls", C.c_longlong), ("contour_steps", C.c_longlong),
                ("kernel_launches", C.c_longlong), ("props_seconds", C.c_double)]


# every symbol include/scft_b200.h declares
EXPORTS = [
    "scft_create", "scft_destroy", "scft_last_error", "scft_status_string", "scft_set_fields",
    "scft_get_fields", "scft_get_conc", "scft_get_doiis", "scft_props", "scft_props_host",
    "scft_do_step", "scft_get_propagator", "scft_solve_field0", "scft_solve_field0_all",
    "scft_solve_field", "scft_string_begin", "scft_string_step", "scft_string_end",
    "scft_free_energy", "scft_last_free_energy", "scft_spline_derivs", "scft_spline_redist", "scft_get_stats",
    "scft_reset_stats", "scft_timer_mark", "scft_timer_elapsed", "scft_set_box", "scft_get_box",
    "scft_stress", "scft_dF_dchi", "scft_relax_cell", "scft_do_step_noalloc",
    "scft_anderson_solve", "scft_autotune", "scft_stress_ckpt", "scft_dF_df",
    "scft_save_checkpoint", "scft_load_checkpoint", "scft_set_box_replica", "scft_get_box_replica",
    "scft_gradients", "scft_props_ckpt", "scft_checkpoint_info", "scft_string_resume",
    "scft_selftest_timeout", "scft_copy_fields", "scft_autotune_ex",
]

_lib = None


def lib():
    """Loads libscft_b200.so (raises ScftError when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ScftError(6, f"{LIB_PATH} is not built (run __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.scft_create.argtypes = [C.POINTER(Problem), C.POINTER(vp)]
    L.scft_destroy.argtypes = [vp]
    L.scft_destroy.restype = None
    L.scft_last_error.argtypes = [vp]
    L.scft_last_error.restype = C.c_char_p
    L.scft_status_string.argtypes = [C.c_int]
    L.scft_status_string.restype = C.c_char_p
    L.scft_set_fields.argtypes = [vp, C.c_int, _dp]
    L.scft_get_fields.argtypes = [vp, C.c_int, _dp]
    L.scft_get_conc.argtypes = [vp, C.c_int, _dp, _dp, _dp]
    L.scft_get_doiis.argtypes = [vp, _ip]
    L.scft_props.argtypes = [vp, C.c_int]
    L.scft_props_host.argtypes = [vp, _dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double, _dp,
                                  C.c_double]
    L.scft_do_step.argtypes = [vp, C.c_int, _dp, _dp, C.c_int]
    L.scft_get_propagator.argtypes = [vp, C.c_int, C.c_int, C.c_int, _dp]
    L.scft_solve_field0.argtypes = [vp, C.c_int, C.c_int, C.c_double, _ip]
    L.scft_solve_field0_all.argtypes = [vp, C.c_int, C.c_double, _ip]
    L.scft_solve_field.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.POINTER(IterReport), _dp,
                                   _dp, _ip]
    L.scft_string_begin.argtypes = [vp, C.c_int, C.c_int, C.c_double]
    L.scft_string_step.argtypes = [vp, C.POINTER(IterReport), _dp, _dp, _ip]
    L.scft_string_end.argtypes = [vp, _ip]
    L.scft_string_resume.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.c_int]
    L.scft_selftest_timeout.argtypes = [vp, C.c_int]
    L.scft_copy_fields.argtypes = [vp, vp]
    L.scft_free_energy.argtypes = [vp, _dp, _dp, _dp, _dp, _dp, _dp]
    L.scft_last_free_energy.argtypes = [vp, _dp, _dp, _dp, _dp, _dp, _dp]
    L.scft_spline_derivs.argtypes = [vp, _dp, C.POINTER(_dp), C.c_int, C.c_int, _ip,
                                     C.POINTER(_dp)]
    L.scft_spline_redist.argtypes = [vp, _dp, _dp, C.POINTER(_dp), C.c_int, C.c_int, _ip,
                                     C.c_double]
    L.scft_get_stats.argtypes = [vp, C.POINTER(Stats)]
    L.scft_reset_stats.argtypes = [vp]
    L.scft_timer_mark.argtypes = [vp, C.c_int]
    L.scft_set_box.argtypes = [vp, _dp]
    L.scft_get_box.argtypes = [vp, _dp]
    L.scft_stress.argtypes = [vp, C.c_int, _dp, _dp]
    L.scft_dF_dchi.argtypes = [vp, C.c_int, _dp]
    L.scft_do_step_noalloc.argtypes = [_ip, _dp, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_int, C.c_void_p]
    L.scft_anderson_solve.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_double, _ip, _dp]
    L.scft_relax_cell.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _ip, _dp]
    L.scft_timer_elapsed.argtypes = [vp, C.c_int, C.c_int, _dp]
    L.scft_autotune.argtypes = [vp, _ip, _ip, _dp]
    L.scft_autotune_ex.argtypes = [vp, _ip, _ip, _ip, _dp]
    L.scft_stress_ckpt.argtypes = [vp, C.c_int, C.c_int, _dp, _dp, _dp]
    L.scft_dF_df.argtypes = [vp, C.c_int, _dp, _dp]
    L.scft_save_checkpoint.argtypes = [vp, C.c_char_p]
    L.scft_set_box_replica.argtypes = [vp, C.c_int, _dp]
    L.scft_gradients.argtypes = [vp, C.c_int, _dp, _dp, _dp]
    L.scft_props_ckpt.argtypes = [vp, C.c_int, C.c_int, _dp, _dp, _dp]
    L.scft_get_box_replica.argtypes = [vp, C.c_int, _dp]
    L.scft_load_checkpoint.argtypes = [vp, C.c_char_p]
    L.scft_checkpoint_info.argtypes = [C.c_char_p, _ip, _ip, _ip, _dp]
    _lib = L
    return L


def _p(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _ptrs(rows):
    arr = (_dp * len(rows))()
    for i, r in enumerate(rows):
        arr[i] = _p(r)
    return arr


class Context:
    """An scft_ctx: every replica of one problem resident on one B200."""

    def __init__(self, m, D, N, chi, f, phidb, ens=2, alpha=0.1, strn=1, fix=(0, 0),
                 dostring=1, springsteps=0, precision="fp64", batched=True, device=0, fcont=0, nostore=0,
                 ckpt_K=0):
        p = Problem()
        p.m = (C.c_int * 3)(*[int(v) for v in m])
        p.D = (C.c_double * 3)(*[float(v) for v in D])
        p.N, p.alpha, p.ens, p.phidb = int(N), float(alpha), int(ens), float(phidb)
        p.chi, p.f, p.strn = float(chi), float(f), int(strn)
        p.fix = (C.c_int * 2)(*[int(v) for v in fix])
        p.dostring, p.springsteps = int(dostring), int(springsteps)
        p.precision = SCFT_FP32 if str(precision).lower() in ("fp32", "float32", "1") else SCFT_FP64
        p.batched = 1 if batched else 0
        p.device = int(device)
        p.fcont = int(fcont)
        p.nostore = int(nostore)
        p.ckpt_K = int(ckpt_K)
        self.problem = p
        self.m = tuple(int(v) for v in m)
        self.M = int(np.prod(self.m))
        self.strn = int(strn)
        self.N = int(N)
        h = C.c_void_p()
        rc = lib().scft_create(C.byref(p), C.byref(h))
        if rc != 0:
            raise ScftError(rc, "scft_create failed")
        self.h = h

    def close(self):
        """Destroys the context (scft_destroy; the reference's `delete D2`)."""
        if getattr(self, "h", None):
            lib().scft_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _ck(self, rc):
        if rc != 0:
            msg = lib().scft_last_error(self.h)
            raise ScftError(rc, msg.decode() if msg else "")

    # fields --------------------------------------------------------------
    def set_fields(self, ii, wm, wp):
        """Replica ii's W- and W+ (M each): the first 2M entries of the reference's
        W[ii] (scft.cu:1037-1051, 1062)."""
        w = np.ascontiguousarray(np.concatenate([np.ravel(wm), np.ravel(wp)]), np.float64)
        self._ck(lib().scft_set_fields(self.h, int(ii), _p(w)))

    def get_fields(self, ii, out=None):
        """[W-, W+] of replica ii; `out` (2M float64, contiguous, may be pinned) is filled in place."""
        w = np.zeros(2 * self.M) if out is None else out
        self._ck(lib().scft_get_fields(self.h, int(ii), _p(w)))
        return w

    def set_fields_2m(self, ii, w2m):
        """Replica ii's [W-, W+] from one contiguous 2M array (no staging copy)."""
        self._ck(lib().scft_set_fields(self.h, int(ii), _p(w2m)))

    def copy_fields_from(self, other):
        """Fields and boxes of every replica of context `other` (same grid and
        replica count), device to device."""
        self._ck(lib().scft_copy_fields(self.h, other.h))

    def get_conc(self, ii):
        """(concentrations [phiA, phiB, phih, phicB] as 4M doubles, lnQ, phis[5]) of
        replica ii's last props: W[ii][2M:6M), lnQ and phis of density::props
        (density.h:344-459)."""
        c = np.zeros(4 * self.M)
        lnQ = C.c_double()
        phis = np.zeros(5)
        self._ck(lib().scft_get_conc(self.h, int(ii), _p(c), C.byref(lnQ), _p(phis)))
        return c, lnQ.value, phis

    def doiis(self):
        """Replica ownership mask of the single process (scft.cu:953-975): 1 for
        every replica, 0 for the fixed ends when fix is set (scft.cu:587-588)."""
        d = np.zeros(self.strn, np.int32)
        self._ck(lib().scft_get_doiis(self.h, d.ctypes.data_as(_ip)))
        return d

    # density -------------------------------------------------------------
    def props(self, ii):
        """density::props (density.h:344-459) of replica ii on its device-resident
        fields; results via get_conc(ii)."""
        self._ck(lib().scft_props(self.h, int(ii)))

    def props_host(self, w, Ns, alpha, phic, f, ii=0):
        """density::props with the reference signature: w (>= 6M doubles) in/out."""
        lnQ = C.c_double()
        phis = np.zeros(5)
        self._ck(lib().scft_props_host(self.h, _p(w), C.byref(lnQ), int(ii), int(Ns), float(alpha),
                                       float(phic), _p(phis), float(f)))
        return lnQ.value, phis

    def do_step(self, ii, qin, s):
        """One Richardson contour step (step::do_step, density.h:129-220) of the
        slice qin = [q(s), q^dagger(s)] (2M doubles) in replica ii's fields;
        returns [q(s+1), q^dagger(s+1)]."""
        qin = np.ascontiguousarray(qin, np.float64).reshape(-1)
        out = np.zeros(2 * self.M)
        self._ck(lib().scft_do_step(self.h, int(ii), _p(qin), _p(out), int(s)))
        return out

    def propagator(self, ii, which, s):
        """Slice s of replica ii's last props: which 0 = q(s), 1 = q^dagger(s)
        (the reference's dev_qq, density.h:368-385)."""
        out = np.zeros(self.M)
        self._ck(lib().scft_get_propagator(self.h, int(ii), int(which), int(s), _p(out)))
        return out

    # solvers -------------------------------------------------------------
    def solve_field0(self, ii, maxIter, errTol):
        """W+ relaxation of replica ii (solve_field0, scft.cu:516-554); returns
        the reference's final k."""
        k = C.c_int()
        self._ck(lib().scft_solve_field0(self.h, int(ii), int(maxIter), float(errTol), C.byref(k)))
        return k.value

    def solve_field0_all(self, maxIter=5000, errTol=1e-4):
        """W+ relaxation of every replica, the prelude of main (scft.cu:1105);
        returns k per replica."""
        k = np.zeros(self.strn, np.int32)
        self._ck(lib().scft_solve_field0_all(self.h, int(maxIter), float(errTol),
                                             k.ctypes.data_as(_ip)))
        return k

    def solve_field(self, maxIter, errTol=1e-3, doii=-1):
        """solve_field (scft.cu:559-809), doii = -1 for the whole string; returns
        (iterations run, per-iteration records, errs and errs3 per iteration and
        replica)."""
        n = max(1, int(maxIter))
        reps = (IterReport * n)()
        errs = np.zeros(n * self.strn)
        errs3 = np.zeros(n * self.strn)
        k = C.c_int()
        self._ck(lib().scft_solve_field(self.h, int(doii), int(maxIter), float(errTol), reps,
                                        _p(errs), _p(errs3), C.byref(k)))
        k = k.value
        recs = [dict(k=r.k, lam=r.lam, errtot=r.errtot, fitup=r.fitup, stepav=r.stepav,
                     did_freee=r.did_freee, FE=r.FE) for r in reps[:k]]
        return k, recs, errs[: k * self.strn].reshape(k, self.strn), \
            errs3[: k * self.strn].reshape(k, self.strn)

    def string_begin(self, maxIter, errTol=1e-3, doii=-1):
        """Starts solve_field one iteration at a time (see string_step)."""
        self._ck(lib().scft_string_begin(self.h, int(doii), int(maxIter), float(errTol)))

    def string_resume(self, k0, maxIter, errTol=1e-3, doii=-1):
        """string_begin with the iteration counter at k0: continues a run from
        fields saved at iteration k0 with the same FreeE cadence."""
        self._ck(lib().scft_string_resume(self.h, int(doii), int(maxIter), float(errTol), int(k0)))

    def string_step(self):
        """One iteration of the solve_field loop (scft.cu:592-806): its record,
        errs, errs3 and whether the loop would stop."""
        rep = IterReport()
        errs = np.zeros(self.strn)
        errs3 = np.zeros(self.strn)
        done = C.c_int()
        self._ck(lib().scft_string_step(self.h, C.byref(rep), _p(errs), _p(errs3), C.byref(done)))
        return dict(k=rep.k, lam=rep.lam, errtot=rep.errtot, fitup=rep.fitup, stepav=rep.stepav,
                    did_freee=rep.did_freee, FE=rep.FE, errs=errs, errs3=errs3,
                    done=bool(done.value))

    def string_end(self):
        """Ends the iteration-at-a-time solve; returns the reference's final k."""
        k = C.c_int()
        self._ck(lib().scft_string_end(self.h, C.byref(k)))
        return k.value

    def free_energy(self):
        """FreeE (scft.cu:812-853): total FE and, per replica, FEs, FEs0, FEs1,
        phctot and the arc-length coordinate alf."""
        s = self.strn
        FE = C.c_double()
        FEs, F0, F1, ph, alf = (np.zeros(s) for _ in range(5))
        self._ck(lib().scft_free_energy(self.h, C.byref(FE), _p(FEs), _p(F0), _p(F1), _p(ph),
                                        _p(alf)))
        return dict(FE=FE.value, FEs=FEs, FEs0=F0, FEs1=F1, phctot=ph, alf=alf)

    def spline_derivs(self, x, Wm, doiis):
        """density::splineDerivsChunked (density.h:491-508) over the whole grid:
        dW-/dalpha of every replica at its knot x[ii] (rows of Wm: W- per
        replica)."""
        strn, M = Wm.shape
        Wm = np.ascontiguousarray(Wm, np.float64)
        out = np.zeros((strn, M))
        d = np.ascontiguousarray(doiis, np.int32)
        self._ck(lib().scft_spline_derivs(self.h, _p(np.ascontiguousarray(x, np.float64)),
                                          _ptrs([Wm[i] for i in range(strn)]), 0, M,
                                          d.ctypes.data_as(_ip), _ptrs([out[i] for i in range(strn)])))
        return out

    def spline_redist(self, x, xref, Wm, doiis, lam):
        """density::splineRedistChunked (density.h:511-528) over the whole grid:
        returns a copy of Wm with interior replicas (doiis == 1) relaxed by lam
        towards the spline at xref."""
        strn, M = Wm.shape
        Wm = np.ascontiguousarray(Wm, np.float64).copy()
        d = np.ascontiguousarray(doiis, np.int32)
        self._ck(lib().scft_spline_redist(self.h, _p(np.ascontiguousarray(x, np.float64)),
                                          _p(np.ascontiguousarray(xref, np.float64)),
                                          _ptrs([Wm[i] for i in range(strn)]), 0, M,
                                          d.ctypes.data_as(_ip), float(lam)))
        return Wm

    def stats(self):
        """Counters of the context: props calls, contour steps, kernel launches
        and device seconds in props rounds (no reference counterpart)."""
        st = Stats()
        self._ck(lib().scft_get_stats(self.h, C.byref(st)))
        return dict(props_calls=st.props_calls, contour_steps=st.contour_steps,
                    kernel_launches=st.kernel_launches, props_seconds=st.props_seconds)

    def reset_stats(self):
        """Zeroes the counters of stats()."""
        self._ck(lib().scft_reset_stats(self.h))

    def set_box(self, D, ii=None):
        """Box of every replica, or of replica ii only."""
        D = np.ascontiguousarray(D, np.float64)
        if ii is None:
            self._ck(lib().scft_set_box(self.h, _p(D)))
        else:
            self._ck(lib().scft_set_box_replica(self.h, int(ii), _p(D)))

    def get_box(self, ii=None):
        """Box lengths D[3] of the context, or of replica ii (the reference's D,
        default 4 4 4 at scft.cu:917)."""
        D = np.zeros(3)
        if ii is None:
            self._ck(lib().scft_get_box(self.h, _p(D)))
        else:
            self._ck(lib().scft_get_box_replica(self.h, int(ii), _p(D)))
        return D

    def stress(self, ii=0):
        """(d lnQ/dL, dF/dL) of replica ii at its current fields (adjoint)."""
        a, b = np.zeros(3), np.zeros(3)
        self._ck(lib().scft_stress(self.h, int(ii), _p(a), _p(b)))
        return a, b

    def props_ckpt(self, ii=0, K=13):
        """density::props of replica ii with propagators kept every K steps;
        returns (lnQ, phis, device bytes); densities as get_conc(ii)."""
        q = C.c_double()
        phis = np.zeros(5)
        nb = C.c_double()
        self._ck(lib().scft_props_ckpt(self.h, int(ii), int(K), C.byref(q), _p(phis), C.byref(nb)))
        return q.value, phis, nb.value

    def stress_ckpt(self, ii=0, K=13):
        """(d lnQ/dL, dF/dL, device bytes) by the adjoint with checkpoints K steps apart."""
        a, b = np.zeros(3), np.zeros(3)
        nb = C.c_double()
        self._ck(lib().scft_stress_ckpt(self.h, int(ii), int(K), _p(a), _p(b), C.byref(nb)))
        return a, b, nb.value

    def anderson_solve(self, ii=0, maxIter=2000, tol=1e-10, nhist=10, lam=0.1):
        """Anderson-mixing solve of replica ii; returns (iterations, RMS residual)."""
        n = C.c_int()
        e = C.c_double()
        self._ck(lib().scft_anderson_solve(self.h, int(ii), int(maxIter), float(tol), int(nhist), float(lam),
                                           C.byref(n), C.byref(e)))
        return n.value, e.value

    def relax_cell(self, ii=0, maxOuter=50, inner=20, stressTol=1e-6, gamma=1.0):
        """Variable-cell relaxation; returns (rounds, last dF/dL, box)."""
        n = C.c_int()
        st = np.zeros(3)
        self._ck(lib().scft_relax_cell(self.h, int(ii), int(maxOuter), int(inner), float(stressTol),
                                       float(gamma), C.byref(n), _p(st)))
        return n.value, st, self.get_box(ii)

    def dF_df(self, ii=0):
        """(d lnQ/df, dF/df) of replica ii; the context needs fcont=1."""
        a, b = C.c_double(), C.c_double()
        self._ck(lib().scft_dF_df(self.h, int(ii), C.byref(a), C.byref(b)))
        return a.value, b.value

    def gradients(self, ii=0):
        """(dF/dL [3], dF/dchiN, dF/df) of replica ii; dF/df is NaN unless fcont=1."""
        dL = np.zeros(3)
        dchi, df = C.c_double(), C.c_double()
        self._ck(lib().scft_gradients(self.h, int(ii), _p(dL), C.byref(dchi), C.byref(df)))
        return dL, dchi.value, df.value

    def dF_dchi(self, ii=0):
        """dF/d(chi N) of replica ii at a converged saddle point:
        1/4 - <W-^2>/chi^2 (no reference counterpart)."""
        v = C.c_double()
        self._ck(lib().scft_dF_dchi(self.h, int(ii), C.byref(v)))
        return v.value

    def autotune(self):
        """(slot groups kept, wide pencil tiles kept, persistent step launch kept,
        best props-round times in ms indexed gi + 3 wide + 6 persistent with
        gi = 0, 1, 2 for 1, 2, 4 slot groups; -1 where not available)."""
        g, w, p = C.c_int(), C.c_int(), C.c_int()
        t = np.zeros(12)
        self._ck(lib().scft_autotune_ex(self.h, C.byref(g), C.byref(w), C.byref(p), _p(t)))
        return g.value, w.value, p.value, [float(v) for v in t]

    def save_checkpoint(self, path):
        """Binary FP64 checkpoint of box and fields of every replica."""
        self._ck(lib().scft_save_checkpoint(self.h, os.fsencode(path)))

    def load_checkpoint(self, path):
        """Boxes and fields of every replica from a binary checkpoint (hash,
        grid and replica count checked)."""
        self._ck(lib().scft_load_checkpoint(self.h, os.fsencode(path)))

    def selftest_timeout(self, polls=1000):
        """Status code of one bounded device wait that nothing completes
        (SCFT_TIMEOUT = 4 expected); the context stays usable."""
        return int(lib().scft_selftest_timeout(self.h, int(polls)))

    def timer_mark(self, slot):
        """Records CUDA event `slot` on the context's stream."""
        self._ck(lib().scft_timer_mark(self.h, int(slot)))

    def timer_elapsed_ms(self, a, b):
        """Device milliseconds between timer slots a and b (waits for b)."""
        ms = C.c_double()
        self._ck(lib().scft_timer_elapsed(self.h, int(a), int(b), C.byref(ms)))
        return ms.value


class Density:
    """``density(Ns, D)`` of the reference (density.h:272) on one B200:
    ``props(w, Ns, alpha, phic, f)`` fills w[2M:6M) and returns (lnQ, phis)."""

    def __init__(self, m, D, Ns, ens, alpha, phic, f, chi=0.0, precision="fp64"):
        self.ctx = Context(m, D, Ns, chi=chi, f=f, phidb=phic, ens=ens, alpha=alpha, strn=1,
                           dostring=0, precision=precision)
        self.M = self.ctx.M

    def props(self, w, Ns, alpha, phic, f):
        """density::props with the reference signature (density.h:344): w[0:2M)
        in, w[2M:6M) out; returns (lnQ, phis)."""
        return self.ctx.props_host(w, Ns, alpha, phic, f)


def checkpoint_info(path) -> dict:
    """Header of a checkpoint file (version, replica count, grid, common box),
    checked as a load checks it; needs no device.  Raises ScftError for a file
    that a load would refuse."""
    v, n = C.c_int(0), C.c_int(0)
    m = (C.c_int * 3)()
    D = np.zeros(3)
    rc = lib().scft_checkpoint_info(os.fsencode(path), C.byref(v), C.byref(n), m, _p(D))
    if rc != 0:
        raise ScftError(rc, f"scft_checkpoint_info: {lib().scft_status_string(rc).decode()}: {path}")
    return {"version": v.value, "strn": n.value, "m": (m[0], m[1], m[2]), "D": tuple(float(x) for x in D)}


def StringSolver(cfg: dict, precision="fp64", batched=True, springsteps=0, device=0) -> Context:
    """A Context for a workload dictionary (see ``scft_string_b200.configs``)."""
    return Context(cfg["m"], cfg["D"], cfg["N"], chi=cfg["chi"], f=cfg["f"], phidb=cfg["phidb"],
                   ens=cfg["ens"], alpha=cfg.get("alpha", 0.1), strn=cfg["strn"],
                   fix=cfg.get("fix", (0, 0)), dostring=cfg.get("dostring", 1),
                   springsteps=springsteps, precision=precision, batched=batched, device=device,
                   fcont=cfg.get("fcont", 0), nostore=cfg.get("nostore", 0), ckpt_K=cfg.get("ckpt_K", 0))
