"""Python binding of the oracle (test infrastructure only).

Loaded by tests/, the smoke check and bench.py's cpu_baseline leg — as the
checker or the timed CPU baseline, never on the product path.  The oracle
is an FP64 C++ restatement of the reference's CPU path; see oracle_core.hpp.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from forcesmith_b200.abi import Session, _dp, _ip, FsError, FS_OK

from . import build as _build

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = _build.build()
        _LIB = C.CDLL(path)
        L = _LIB
        L.orc_create.argtypes = [C.POINTER(C.c_void_p)]
        for name in ("destroy", "prepare"):
            getattr(L, f"orc_{name}").argtypes = [C.c_void_p]
        L.orc_eval_jacobian_fd.argtypes = [C.c_void_p, C.c_double, C.c_double,
                                           C.POINTER(C.c_double), C.c_int32, C.c_int32]
        L.orc_eval_jacobian_analytic.argtypes = [C.c_void_p, C.c_double, C.c_double,
                                                 C.POINTER(C.c_double)]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_normal_equations.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double),
                                           C.c_int64, C.c_int32, C.POINTER(C.c_double),
                                           C.POINTER(C.c_double)]
        L.orc_lm_step.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int32,
                                  C.c_double, C.c_int32, C.POINTER(C.c_double)]
        L.orc_lsq_step.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int32,
                                   C.c_double, C.POINTER(C.c_double)]
        L.orc_eval_population.argtypes = [C.c_void_p, C.c_double, C.c_double,
                                          C.POINTER(C.c_double), C.c_int32,
                                          C.POINTER(C.c_double)]
        L.orc_spline_eval.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int32,
                                      C.c_double, C.POINTER(C.c_double)]
        L.orc_spline_slopes.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int32,
                                        C.POINTER(C.c_double)]
        L.orc_spline_grad.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int32,
                                      C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double)]
        L.orc_form_eval.argtypes = [C.c_int32, C.POINTER(C.c_double), C.c_int32, C.c_double,
                                    C.POINTER(C.c_double), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.c_double]
        L.orc_pbc.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double),
                              C.POINTER(C.c_double), C.POINTER(C.c_double),
                              C.POINTER(C.c_double)]
        L.orc_residual_count.argtypes = [C.c_void_p, C.c_double, C.POINTER(C.c_int64)]
        L.orc_eval.argtypes = [C.c_void_p, C.c_double, C.c_double] + [C.POINTER(C.c_double)] * 6
        L.orc_set_params.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int32]
        L.orc_acsf_standardization.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                               C.POINTER(C.c_int64)]
        L.orc_descriptor.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double)]
    return _LIB


def set_threads(n: int) -> int:
    return lib().orc_set_threads(n)


class Oracle(Session):
    """FP64 CPU restatement with the same call set as the device library."""

    def __init__(self):
        L = lib()
        h = C.c_void_p()
        rc = L.orc_create(C.byref(h))
        if rc != FS_OK:
            raise FsError(rc, "orc_create")
        super().__init__(L, "orc", h)

    def __del__(self):
        try:
            if self._h:
                self._lib.orc_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def neighbors(self):
        P = self.num_pairs()
        j = np.zeros(P, np.int32)
        img = np.zeros(3 * P, np.int8)
        d = np.zeros(3 * P, np.float64)
        rc = self._lib.orc_get_neighbors(self._h, _ip(j), img.ctypes.data_as(C.POINTER(C.c_int8)),
                                         _dp(d))
        self._check(rc, "get_neighbors")
        return j, img.reshape(-1, 3), d.reshape(-1, 3)

    def descriptor(self, c, i, size):
        """Descriptor values of atom i of configuration c (ACSF or LMBTR)."""
        D = np.zeros(size, np.float64)
        self._check(self._lib.orc_descriptor(self._h, c, i, _dp(D)), "descriptor")
        return D

    def jacobian_fd(self, w_e=1.0, w_s=0.0, c0=0, c1=-1):
        m = self.residual_count(w_s)
        J = np.zeros((self.D, m))  # column-major m×D == row-major D×m
        rc = self._lib.orc_eval_jacobian_fd(self._h, w_e, w_s, _dp(J), c0, c1)
        self._check(rc, "eval_jacobian_fd")
        return J.T  # m × D view

    def jacobian_analytic(self, w_e=1.0, w_s=0.0):
        m = self.residual_count(w_s)
        J = np.zeros((self.D, m))
        rc = self._lib.orc_eval_jacobian_analytic(self._h, w_e, w_s, _dp(J))
        self._check(rc, "eval_jacobian_analytic")
        return J.T

    def eval_population(self, xs, w_e=1.0, w_s=0.0):
        xs = np.ascontiguousarray(xs, np.float64)
        obj = np.zeros(xs.shape[0])
        rc = self._lib.orc_eval_population(self._h, w_e, w_s, _dp(xs), xs.shape[0], _dp(obj))
        self._check(rc, "eval_population")
        return obj


def normal_equations(J, F):
    """JᵀJ and Jᵀr in FP64 from an m × D Jacobian."""
    Jc = np.asfortranarray(J)  # column-major
    m, D = Jc.shape
    JtJ = np.zeros((D, D))
    Jtr = np.zeros(D)
    F = np.ascontiguousarray(F, np.float64)
    lib().orc_normal_equations(Jc.ctypes.data_as(C.POINTER(C.c_double)), _dp(F), m, D,
                               _dp(JtJ), _dp(Jtr))
    return JtJ, Jtr


def lm_step(JtJ, Jtr, lam, mode=0):
    D = Jtr.size
    dx = np.zeros(D)
    rc = lib().orc_lm_step(_dp(np.ascontiguousarray(JtJ)), _dp(np.ascontiguousarray(Jtr)), D,
                           lam, mode, _dp(dx))
    if rc != FS_OK:
        raise FsError(rc, "orc_lm_step")
    return dx


def lsq_step(JtJ, Jtr, ridge=0.0):
    D = Jtr.size
    dx = np.zeros(D)
    rc = lib().orc_lsq_step(_dp(np.ascontiguousarray(JtJ)), _dp(np.ascontiguousarray(Jtr)), D,
                            ridge, _dp(dx))
    if rc != FS_OK:
        raise FsError(rc, "orc_lsq_step")
    return dx


def spline_eval(x, y, r):
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    out = np.zeros(6)
    lib().orc_spline_eval(_dp(x), _dp(y), x.size, r, _dp(out))
    return out  # eval, deriv, eval_at, deriv_at, deriv2, interval


def spline_slopes(x, y):
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    s = np.zeros(x.size)
    lib().orc_spline_slopes(_dp(x), _dp(y), x.size, _dp(s))
    return s


def spline_grad(x, y, r):
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    gv, gd, gdd = np.zeros(x.size), np.zeros(x.size), np.zeros(x.size)
    lib().orc_spline_grad(_dp(x), _dp(y), x.size, r, _dp(gv), _dp(gd), _dp(gdd))
    return gv, gd, gdd


def form_eval(form, params, r, rmax=0.0):
    """Value, d/dr, d²/dr² and the parameter partials ∂v/∂θ, ∂²v/∂r∂θ of an
    analytic form at r; rmax is the table's upper gate bound (the switching
    point of the smooth-cutoff forms)."""
    p = np.ascontiguousarray(params, np.float64)
    out = np.zeros(3)
    g, dg = np.zeros(p.size), np.zeros(p.size)
    rc = lib().orc_form_eval(form, _dp(p), p.size, r, _dp(out), _dp(g), _dp(dg), rmax)
    if rc != FS_OK:
        raise FsError(rc, "orc_form_eval")
    return out, g, dg


def pbc(box9, r3=None):
    b = np.ascontiguousarray(box9, np.float64).reshape(9)
    r = np.zeros(3) if r3 is None else np.ascontiguousarray(r3, np.float64)
    w, vol, inv = np.zeros(3), C.c_double(), np.zeros(9)
    lib().orc_pbc(_dp(b), _dp(r), _dp(w), C.byref(vol), _dp(inv))
    return w, vol.value, inv.reshape(3, 3)
