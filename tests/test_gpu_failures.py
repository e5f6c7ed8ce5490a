"""Failure detection on the device, in the forms that fault no GPU.

- A bounded wait that runs out: fs_gpu_check_bounded_wait makes one CTA wait,
  with a short cycle budget and the tensor-core kernels' own wait routine,
  on a barrier phase that nothing completes (no copy or MMA bound to it).
  The call must return FS_ERR_DEVICE, and the context must stay usable: the
  next evaluation succeeds and matches the one before.
- Non-finite input injected on the host: fs_gpu_set_params refuses a NaN
  parameter vector with FS_ERR_NUMERIC and keeps the model; a NaN trial
  vector in a population gives a NaN objective in its own row only.
- A normal-equation matrix that is not positive definite (the singular
  undamped matrix of a model with a species absent from the data) makes
  fs_gpu_lm_step return FS_ERR_NUMERIC; a negative damping is refused as an
  argument error before any solve.
"""
import numpy as np
import pytest

from forcesmith_b200 import synth
from forcesmith_b200.abi import FS_ERR_ARG, FS_ERR_DEVICE, FS_ERR_NUMERIC, FsError
from tests.helpers import small_ternary, ternary_models

pytestmark = pytest.mark.gpu


def _session(precision="fp32"):
    from forcesmith_b200.gpu import GpuSession
    true, start = ternary_models(12)
    ds = small_ternary(3, 40, seed=5)
    g = GpuSession(0, precision)
    g.upload(ds)
    g.set_model(start)
    return g


def test_bounded_wait_gives_up_and_context_survives():
    g = _session()
    before = g.eval(1.0, 0.1)
    rc = g._lib.fs_gpu_check_bounded_wait(g._h, 200000)  # ≈ 0.1 ms at 2 GHz
    assert rc == FS_ERR_DEVICE
    assert "timed out" in g.last_error()
    after = g.eval(1.0, 0.1)  # the error word was reset; the context works
    assert np.array_equal(after["F"], before["F"])
    rc = g._lib.fs_gpu_check_bounded_wait(g._h, 0)
    assert rc != 0 and rc != FS_ERR_DEVICE  # a budget outside [1, 4e9] is an argument error


def test_nan_parameters_refused_and_model_kept():
    g = _session("fp64")
    x = g.gather_params()
    ref = g.eval(1.0, 0.1)["obj"]
    bad = x.copy()
    bad[7] = np.nan
    with pytest.raises(FsError) as e:
        g.set_params(bad)
    assert e.value.code == FS_ERR_NUMERIC and "parameter 7" in str(e.value)
    bad[7] = np.inf
    with pytest.raises(FsError):
        g.set_params(bad)
    assert np.array_equal(g.gather_params(), x)
    assert g.eval(1.0, 0.1)["obj"] == ref


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_nan_trial_vector_stays_in_its_row(precision):
    g = _session(precision)
    x = g.gather_params()
    xs = np.stack([x * synth.uniform(x.size, 0.98, 1.02, 50 + k) for k in range(6)])
    clean = g.eval_population(xs, 1.0, 0.1)
    xs[2, :] = np.nan
    got = g.eval_population(xs, 1.0, 0.1)
    assert np.isnan(got[2])
    rest = [0, 1, 3, 4, 5]
    assert np.array_equal(got[rest], clean[rest])


def test_lm_step_not_positive_definite():
    g = _session("fp64")
    res = g.jacobian(1.0, 0.1, want_J=False)
    scale = float(np.max(np.diag(res["JtJ"])))
    with pytest.raises(FsError) as e:
        g.lm_step(-10.0 * scale, 0)
    assert e.value.code == FS_ERR_ARG
    # a species slot absent from the data: its density and embedding columns
    # are zero, so the undamped JᵀJ is singular
    from forcesmith_b200.gpu import GpuSession
    true, start = ternary_models(12)
    ds = small_ternary(2, 40, seed=5)
    ds.type[:] = ds.type % 2
    h = GpuSession(0, "fp64")
    h.upload(ds)
    h.set_model(start)
    r = h.jacobian(1.0, 0.1, want_J=False)
    assert np.any(np.all(r["JtJ"] == 0.0, axis=0))
    with pytest.raises(FsError) as e:
        h.lm_step(0.0, 0)
    assert e.value.code == FS_ERR_NUMERIC
    dx = h.lm_step(1e-3, 0)  # damped: a zero column gets λ on its diagonal
    assert np.all(np.isfinite(dx))
