"""The C++ adapter (include/forcesmith_gpu_adapter.hpp) driven the way
Forcesmith's functor drives a force calculator: prepare() once, then
eval_forces(cfg, c) and eval_cached_jacobian(c, …) from four threads at once
(forcesmith_functor.cpp:43-51, 111-132), then a GpuLMSolver fit.  The
program tests/cpp/adapter_test.cpp is built by tests/cpp/build.py.

Checked against the oracle on a ternary spline EAM case (FP64 context):
forces, energies, stress (already /V) and limits 1e-9·(1 + |x|); the
column-major fjac filled block by block against the oracle's analytic
Jacobian, 1e-9·(1 + |J|); a configuration evaluated on its own equals its
slice of the batch to 1e-12; the C++ LM reproduces the Python LMSolver's
trajectory on the same device (the same arithmetic): objectives per
iteration within 1e-9 relative; the C++ DE run equals the Python DESolver's
with the same seed and generation count (the same device kernels).
"""
import os
import struct
import subprocess

import numpy as np
import pytest

from forcesmith_b200.abi import FS_PREC_FP64
from oracle import api as O
from tests.helpers import label, small_ternary, ternary_models

pytestmark = pytest.mark.gpu

W_E, W_S = 1.0, 0.1
LM_ITERS = 8
DE_GENERATIONS = 20


def _write_case(path, ds, model, x, threads=4):
    with open(path, "wb") as f:
        f.write(struct.pack("<8i", ds.n_cfg, model.family, model.ntypes, len(model.tables), FS_PREC_FP64,
                            threads, LM_ITERS, DE_GENERATIONS))
        a0 = 0
        for c in range(ds.n_cfg):
            n = int(ds.natoms[c])
            f.write(struct.pack("<i", n))
            f.write(np.asarray(ds.box9[c], "<f8").tobytes())
            for i in range(a0, a0 + n):
                f.write(struct.pack("<i", int(ds.type[i])))
                f.write(np.asarray(ds.pos[i], "<f8").tobytes())
                f.write(np.asarray(ds.ref_force[i], "<f8").tobytes())
            f.write(struct.pack("<d", float(ds.ref_energy[c])))
            f.write(np.asarray(ds.ref_stress9[c], "<f8").tobytes())
            a0 += n
        for t in model.tables:
            f.write(struct.pack("<3i2d", t.kind, t.form, t.values.size, t.rmin, t.rmax))
            f.write(np.asarray(t.values, "<f8").tobytes())
        f.write(struct.pack("<2di", W_E, W_S, x.size))
        f.write(np.asarray(x, "<f8").tobytes())


def test_cpp_adapter_against_oracle(tmp_path):
    from tests.cpp.build import build
    from forcesmith_b200 import solvers
    from forcesmith_b200.gpu import GpuSession
    true, start = ternary_models(12)
    ds = label(small_ternary(5, 40, seed=77), true, O.Oracle, W_E, W_S)
    assert all(t.fixed is None or not t.fixed.any() for t in start.tables)  # the case carries no masks
    x = start.free_values() * 1.01
    case, out = tmp_path / "case.bin", tmp_path / "out.bin"
    _write_case(case, ds, start, x)
    exe = build()
    r = subprocess.run([exe, str(case), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = out.read_bytes()
    o = O.Oracle()
    o.upload(ds)
    o.set_model(start)
    o.set_params(x)
    ref = o.eval(W_E, W_S)
    Ja = o.jacobian_analytic(W_E, W_S)
    M, D, N, C = Ja.shape[0], x.size, ds.n_atoms, ds.n_cfg
    off = 0

    def take(n):
        nonlocal off
        a = np.frombuffer(raw, "<f8", n, off)
        off += 8 * n
        return a
    forces = take(3 * N).reshape(-1, 3)
    per_cfg = take(11 * C).reshape(C, 11)
    J = take(M * D).reshape(D, M).T
    solo_f = take(3 * int(ds.natoms[0])).reshape(-1, 3)
    solo_e, solo_s = take(1)[0], take(9)

    def close(a, b, tol, what):
        err = np.max(np.abs(np.asarray(a) - np.asarray(b)) / (1.0 + np.abs(b)))
        assert err <= tol, f"{what}: {err:.3e}"
    close(forces, ref["forces"].reshape(-1, 3), 1e-9, "forces")
    close(per_cfg[:, 0], ref["energy"], 1e-9, "energy")
    close(per_cfg[:, 1:10], ref["stress"].reshape(C, 9), 1e-9, "stress")
    close(per_cfg[:, 10], ref["limit"], 1e-9, "limit")
    close(J, Ja, 1e-9, "fjac")
    n0 = int(ds.natoms[0])
    assert np.allclose(solo_f, forces[:n0], rtol=1e-12, atol=1e-12)
    assert abs(solo_e - per_cfg[0, 0]) <= 1e-12 * abs(per_cfg[0, 0])
    assert np.allclose(solo_s, per_cfg[0, 1:10], rtol=1e-12, atol=1e-15)
    status, iters, nh = struct.unpack_from("<3i", raw, off)
    off += 12
    hist = np.frombuffer(raw, "<f8", nh, off)
    off += 8 * nh
    x_fit = np.frombuffer(raw, "<f8", D, off)
    assert status in (1, 2, 3) and iters >= 1 and hist[-1] < hist[0]
    # the same LM in Python on the same device
    g = GpuSession(0, "fp64")
    g.upload(ds)
    g.set_model(start)
    _, x_py, info = solvers.LMSolver(max_iter=LM_ITERS).minimize(g, x, w_e=W_E, w_s=W_S)
    py = np.asarray(info["obj"])
    assert py.size == hist.size, (py, hist)
    assert np.allclose(hist, py, rtol=1e-9, atol=0.0), (hist, py)
    assert np.allclose(x_fit, x_py, rtol=1e-7, atol=1e-10)
    de_best = struct.unpack_from("<d", raw, off + 8 * D)[0]
    x_de = np.frombuffer(raw, "<f8", D, off + 8 * D + 8)
    assert off + 8 * D + 8 + 8 * D == len(raw)
    _, x_de_py, de_info = solvers.DESolver(max_generations=DE_GENERATIONS).minimize(g, x, w_e=W_E, w_s=W_S)
    assert de_best == pytest.approx(de_info["obj"], rel=1e-12)
    assert np.allclose(x_de, x_de_py, rtol=1e-12, atol=0.0)
    assert de_best <= hist[0] * (1 + 1e-12)  # member 0 starts at x (population-kernel sum order)
