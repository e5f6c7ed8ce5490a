"""ctypes binding of libforcesmith_b200.so (include/forcesmith_gpu.h).

The device library is the only implementation behind this class: if the
shared object is missing or no CUDA device is visible, construction raises —
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .abi import (fs_de_opts, fs_surrogate_opts, fs_table, fs_tune_report, FS_OK, FS_PREC_FP32, FS_PREC_FP64, FsError, Session, _dp, _ip, fs_gpu_opts,
                  fs_model, load_library)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libforcesmith_b200.so")

_LIB = None


def _check_abi(L):
    """The library's struct sizes against these bindings' (a stale build
    would otherwise write past a caller's struct)."""
    ours = [C.sizeof(t) for t in (fs_table, fs_model, fs_gpu_opts, fs_tune_report, fs_de_opts, fs_surrogate_opts)]
    got = (C.c_int64 * 6)()
    L.fs_gpu_abi_sizes.argtypes = [C.POINTER(C.c_int64), C.c_int32]
    if L.fs_gpu_abi_sizes(got, 6) != 6 or list(got) != ours:
        raise ImportError(f"{LIB_PATH} was built against another forcesmith_gpu.h (struct sizes {list(got)}, "
                          f"bindings {ours}); rebuild it with `python -m forcesmith_b200.build`")


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is not built; run `python -m forcesmith_b200.build` (nvcc, sm_100a)")
        L = load_library(LIB_PATH)
        _check_abi(L)
        vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        pd, pi = C.POINTER(C.c_double), C.POINTER(C.c_int32)
        L.fs_gpu_create.argtypes = [C.POINTER(fs_gpu_opts), C.POINTER(vp)]
        L.fs_gpu_destroy.argtypes = [vp]
        L.fs_gpu_last_error.argtypes = [vp, C.c_char_p, C.c_size_t]
        L.fs_gpu_get_stream.argtypes = [vp, C.POINTER(vp)]
        L.fs_gpu_upload_configs.argtypes = [vp, i32, pi, pd, pd, pi, pd, pd, pd]
        L.fs_gpu_set_references.argtypes = [vp, pd, pd, pd]
        L.fs_gpu_set_model.argtypes = [vp, C.POINTER(fs_model)]
        L.fs_gpu_prepare.argtypes = [vp]
        L.fs_gpu_num_pairs.argtypes = [vp, C.POINTER(i64)]
        L.fs_gpu_get_neighbor_counts.argtypes = [vp, pi]
        L.fs_gpu_get_neighbors.argtypes = [vp, pi, C.POINTER(C.c_int8)]
        L.fs_gpu_param_count.argtypes = [vp, pi]
        L.fs_gpu_gather_params.argtypes = [vp, pd]
        L.fs_gpu_gather_bounds.argtypes = [vp, pd, pd]
        L.fs_gpu_set_params.argtypes = [vp, pd, i32]
        L.fs_gpu_residual_count.argtypes = [vp, dbl, C.POINTER(i64)]
        L.fs_gpu_eval.argtypes = [vp, dbl, dbl, pd, pd, pd, pd, pd, pd]
        L.fs_gpu_eval_jacobian.argtypes = [vp, dbl, dbl, pd, pd, pd, pd, pd]
        L.fs_gpu_eval_jacobian_async.argtypes = [vp, dbl, dbl]
        L.fs_gpu_copy_jacobian_rows.argtypes = [vp, i64, i64, pd, i64]
        L.fs_gpu_check_bounded_wait.argtypes = [vp, i64]
        L.fs_gpu_max_cutoff.argtypes = [vp, pd]
        L.fs_gpu_tabulate.argtypes = [vp, C.c_int32, C.c_int32, pd, pd, pd]
        L.fs_gpu_fetch_normal_equations.argtypes = [vp, pd, pd, pd]
        L.fs_gpu_lm_step.argtypes = [vp, dbl, i32, pd]
        L.fs_gpu_lsq_step.argtypes = [vp, dbl, pd]
        L.fs_gpu_acsf_standardization.argtypes = [vp, pd, pd, C.POINTER(C.c_int64)]
        L.fs_gpu_eval_population.argtypes = [vp, dbl, dbl, pd, i32, pd]
        L.fs_gpu_de_init.argtypes = [vp, C.POINTER(fs_de_opts), pd, pd, pd]
        L.fs_gpu_de_run.argtypes = [vp, i32, i32, pd, pd, pd]
        L.fs_gpu_de_population.argtypes = [vp, pd, pd]
        L.fs_gpu_eval_population_noalloc.argtypes = [vp, dbl, dbl, vp, i32, vp]
        L.fs_gpu_autotune.argtypes = [vp, dbl, dbl, C.POINTER(fs_tune_report)]
        pf = C.POINTER(C.c_float)
        L.fs_gpu_surrogate_init.argtypes = [vp, C.POINTER(fs_surrogate_opts)]
        L.fs_gpu_de_run_screened.argtypes = [vp, i32, pd, pd, pd, pd, pi]
        L.fs_gpu_surrogate_param_count.argtypes = [vp, C.POINTER(i64)]
        L.fs_gpu_surrogate_get_params.argtypes = [vp, pf]
        L.fs_gpu_surrogate_set_params.argtypes = [vp, pf]
        L.fs_gpu_surrogate_predict.argtypes = [vp, pf, i32, pf]
        L.fs_gpu_surrogate_gradient.argtypes = [vp, pf, pf, i32, pf, pf]
        L.fs_gpu_surrogate_train.argtypes = [vp, pf, pf, i32, i32, pf]
        _LIB = L
    return _LIB


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _err(h) -> str:
    buf = C.create_string_buffer(512)
    if h:
        lib().fs_gpu_last_error(h, buf, 512)
    return buf.value.decode(errors="replace")


class GpuSession(Session):
    """One fs_gpu context (one device, one stream)."""

    def __init__(self, device: int = 0, precision: str = "fp32", lanes_per_atom: int = 0):
        L = lib()
        opts = fs_gpu_opts(device, FS_PREC_FP64 if precision == "fp64" else FS_PREC_FP32,
                           lanes_per_atom, 0)
        h = C.c_void_p()
        rc = L.fs_gpu_create(C.byref(opts), C.byref(h))
        if rc != FS_OK:
            raise FsError(rc, "fs_gpu_create (is a CUDA device visible?)")
        super().__init__(L, "fs_gpu", h, err_fn=_err)
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fs_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self) -> str:
        """fs_gpu_last_error: the context's last error message."""
        return _err(self._h)

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        self._check(self._lib.fs_gpu_get_stream(self._h, C.byref(s)), "get_stream")
        return s.value or 0

    def neighbors(self):
        P = self.num_pairs()
        j = np.zeros(P, np.int32)
        img = np.zeros(3 * P, np.int8)
        self._check(self._lib.fs_gpu_get_neighbors(self._h, _ip(j),
                                                   img.ctypes.data_as(C.POINTER(C.c_int8))),
                    "get_neighbors")
        return j, img.reshape(-1, 3)

    def jacobian(self, w_e=1.0, w_s=0.0, want_J=True):
        m = self.residual_count(w_s)
        D = self.D
        F = np.zeros(m)
        J = np.zeros((D, m)) if want_J else None  # column-major m × D
        JtJ = np.zeros((D, D))
        Jtr = np.zeros(D)
        obj = C.c_double()
        rc = self._lib.fs_gpu_eval_jacobian(self._h, w_e, w_s, _dp(F), _dp(J), _dp(JtJ), _dp(Jtr),
                                            C.byref(obj))
        self._check(rc, "eval_jacobian")
        return dict(F=F, J=None if J is None else J.T, JtJ=JtJ, Jtr=Jtr, obj=obj.value)

    def jacobian_rows(self, row0, nrows, ld=None):
        """fs_gpu_copy_jacobian_rows: rows [row0, row0 + nrows) of the last
        Jacobian as an FP64 (nrows × D) array, from a column-major block of
        leading dimension ld (default nrows)."""
        ld = nrows if ld is None else ld
        buf = np.full((self.D, ld), np.nan)  # column-major ld × D
        self._check(self._lib.fs_gpu_copy_jacobian_rows(self._h, int(row0), int(nrows), _dp(buf), int(ld)),
                    "copy_jacobian_rows")
        return buf[:, :nrows].T, buf

    def max_cutoff(self):
        """fs_gpu_max_cutoff: the model's interaction cut-off."""
        rc = C.c_double()
        self._check(self._lib.fs_gpu_max_cutoff(self._h, C.byref(rc)), "max_cutoff")
        return rc.value

    def tabulate(self, table, r):
        """fs_gpu_tabulate: (value, d/dr) of radial table `table` at the
        points r, FP64, at the current parameters."""
        r = np.ascontiguousarray(r, np.float64)
        v, dv = np.zeros(r.size), np.zeros(r.size)
        self._check(self._lib.fs_gpu_tabulate(self._h, int(table), int(r.size), _dp(r), _dp(v), _dp(dv)),
                    "tabulate")
        return v, dv

    def jacobian_async(self, w_e=1.0, w_s=0.0):
        self._check(self._lib.fs_gpu_eval_jacobian_async(self._h, w_e, w_s), "eval_jacobian_async")

    def normal_equations(self):
        D = self.D
        JtJ, Jtr, obj = np.zeros((D, D)), np.zeros(D), C.c_double()
        self._check(self._lib.fs_gpu_fetch_normal_equations(self._h, _dp(JtJ), _dp(Jtr),
                                                            C.byref(obj)), "fetch_normal_equations")
        return JtJ, Jtr, obj.value

    def lm_step(self, lam, mode=0):
        dx = np.zeros(self.D)
        self._check(self._lib.fs_gpu_lm_step(self._h, lam, mode, _dp(dx)), "lm_step")
        return dx

    def lsq_step(self, ridge=0.0):
        dx = np.zeros(self.D)
        self._check(self._lib.fs_gpu_lsq_step(self._h, ridge, _dp(dx)), "lsq_step")
        return dx

    def eval_population(self, xs, w_e=1.0, w_s=0.0):
        xs = np.ascontiguousarray(xs, np.float64)
        obj = np.zeros(xs.shape[0])
        self._check(self._lib.fs_gpu_eval_population(self._h, w_e, w_s, _dp(xs), xs.shape[0],
                                                     _dp(obj)), "eval_population")
        return obj

    def autotune(self, w_e=1.0, w_s=0.0):
        """fs_gpu_autotune: time the kernels' launch shapes on this context's
        data and keep the fastest; returns the choices and timings."""
        r = fs_tune_report()
        self._check(self._lib.fs_gpu_autotune(self._h, w_e, w_s, C.byref(r)), "autotune")
        return dict(lanes_per_atom=r.lanes_per_atom, k2_warps=r.k2_warps, pop_waves=r.pop_waves,
                    residual_ms=list(r.residual_ms), jacobian_ms=list(r.jacobian_ms),
                    population_ms=list(r.population_ms))

    def eval_population_noalloc(self, xs_dev_ptr, NP, obj_dev_ptr, w_e=1.0, w_s=0.0):
        """fs_gpu_eval_population_noalloc: objectives of NP trial vectors
        already in device memory (xs_dev_ptr: NP × D doubles) into device
        memory (obj_dev_ptr: NP doubles), with no allocation by the library.
        Asynchronous on this context's stream."""
        self._check(self._lib.fs_gpu_eval_population_noalloc(
            self._h, w_e, w_s, C.c_void_p(xs_dev_ptr), int(NP), C.c_void_p(obj_dev_ptr)),
            "eval_population_noalloc")

    # -- differential evolution on the device ---------------------------------
    def de_init(self, lo, hi, x0=None, NP=None, mutation=0.65, crossover=0.5, seed=42,
                w_e=1.0, w_s=0.0):
        lo = np.ascontiguousarray(lo, np.float64)
        hi = np.ascontiguousarray(hi, np.float64)
        NP = int(NP if NP is not None else 15 * lo.size)
        o = fs_de_opts(NP, 0, float(mutation), float(crossover), int(seed), float(w_e), float(w_s))
        px = None
        if x0 is not None:
            x0 = np.ascontiguousarray(x0, np.float64)
            px = _dp(x0)
        self._check(self._lib.fs_gpu_de_init(self._h, C.byref(o), _dp(lo), _dp(hi), px), "de_init")
        self._de_np = NP

    def de_run(self, generations, use_graph=True, history=False):
        D = self.D
        best = np.zeros(1)
        x = np.zeros(D)
        hist = np.zeros(max(int(generations), 1)) if history else None
        self._check(self._lib.fs_gpu_de_run(self._h, int(generations), 1 if use_graph else 0,
                                            _dp(best), _dp(x), _dp(hist) if history else None),
                    "de_run")
        return (best[0], x, hist[:generations]) if history else (best[0], x)

    # -- surrogate-screened DE ------------------------------------------------
    def surrogate_init(self, screen=4, warm_generations=5, batch=512, steps_per_generation=32,
                       lr=1e-3, gate=0.8, holdout=0.1, seed=1, archive_rows=0):
        o = fs_surrogate_opts(int(screen), int(warm_generations), int(batch),
                              int(steps_per_generation), float(lr), float(gate), float(holdout),
                              int(seed), int(archive_rows))
        self._check(self._lib.fs_gpu_surrogate_init(self._h, C.byref(o)), "surrogate_init")

    def de_run_screened(self, generations):
        g = int(generations)
        best = np.zeros(1)
        x = np.zeros(self.D)
        hist = np.zeros(max(g, 1))
        rho = np.zeros(max(g, 1))
        scr = np.zeros(max(g, 1), np.int32)
        self._check(self._lib.fs_gpu_de_run_screened(self._h, g, _dp(best), _dp(x), _dp(hist),
                                                     _dp(rho), _ip(scr)), "de_run_screened")
        return best[0], x, dict(history=hist[:g], rho=rho[:g], screened=scr[:g].astype(bool))

    def surrogate_params(self):
        n = C.c_int64()
        self._check(self._lib.fs_gpu_surrogate_param_count(self._h, C.byref(n)), "surrogate_param_count")
        p = np.zeros(n.value, np.float32)
        self._check(self._lib.fs_gpu_surrogate_get_params(self._h, _fp(p)), "surrogate_get_params")
        return p

    def surrogate_set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(self._lib.fs_gpu_surrogate_set_params(self._h, _fp(p)), "surrogate_set_params")

    def surrogate_predict(self, X):
        X = np.ascontiguousarray(X, np.float32)
        y = np.zeros(X.shape[0], np.float32)
        self._check(self._lib.fs_gpu_surrogate_predict(self._h, _fp(X), X.shape[0], _fp(y)),
                    "surrogate_predict")
        return y

    def surrogate_gradient(self, X, t):
        X = np.ascontiguousarray(X, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        n = C.c_int64()
        self._check(self._lib.fs_gpu_surrogate_param_count(self._h, C.byref(n)), "surrogate_param_count")
        g = np.zeros(n.value, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(self._lib.fs_gpu_surrogate_gradient(self._h, _fp(X), _fp(t), X.shape[0], _fp(g),
                                                        _fp(loss)), "surrogate_gradient")
        return float(loss[0]), g

    def surrogate_train(self, X, t, steps):
        X = np.ascontiguousarray(X, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(self._lib.fs_gpu_surrogate_train(self._h, _fp(X), _fp(t), X.shape[0], int(steps),
                                                     _fp(loss)), "surrogate_train")
        return float(loss[0])

    def de_population(self):
        D = self.D
        pop = np.zeros((self._de_np, D))
        obj = np.zeros(self._de_np)
        self._check(self._lib.fs_gpu_de_population(self._h, _dp(pop), _dp(obj)), "de_population")
        return pop, obj


def _bind_instrumentation():
    L = lib()
    L.fs_gpu_set_profiling.argtypes = [C.c_void_p, C.c_int32]
    L.fs_gpu_phase_times.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int32,
                                     C.POINTER(C.c_int32)]
    L.fs_gpu_launch_count.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    L.fs_gpu_copy_normal_equations.argtypes = [C.c_void_p, C.c_void_p]


PHASES = ("residual", "jac_atoms", "jac_forces", "gram")


def set_profiling(sess: GpuSession, max_steps: int):
    _bind_instrumentation()
    sess._check(sess._lib.fs_gpu_set_profiling(sess._h, max_steps), "set_profiling")


def phase_times(sess: GpuSession):
    _bind_instrumentation()
    ms = np.zeros(8)
    steps = C.c_int32()
    sess._check(sess._lib.fs_gpu_phase_times(sess._h, _dp(ms), 8, C.byref(steps)), "phase_times")
    return dict(zip(PHASES, ms[:4].tolist())), steps.value


def launch_count(sess: GpuSession) -> int:
    _bind_instrumentation()
    n = C.c_int64()
    sess._check(sess._lib.fs_gpu_launch_count(sess._h, C.byref(n)), "launch_count")
    return n.value


def copy_normal_equations(sess: GpuSession, dst_ptr: int):
    _bind_instrumentation()
    sess._check(sess._lib.fs_gpu_copy_normal_equations(sess._h, C.c_void_p(dst_ptr)),
                "copy_normal_equations")
