"""fs_gpu_eval_population_noalloc — the population objective for callers that
cannot allocate device memory (a host whose GPU memory is all owned by its
own pool, or a loop that must not let cudaMalloc / cudaFree synchronise the
device).  The library's scratch for this call is a fixed 8 MiB device array.

Checked through the C ABI against fs_gpu_eval_population on the same trial
vectors, twice in a row with different sizes (the array keeps the previous
call's contents; a call must not depend on them): the two entry points run
the same kernels, so the bar is relative 1e-12.  Too large an NP is refused
with an error that states the limit, and that limit itself is accepted.
The call allocates nothing: on a fresh context (whose allocating population
buffers do not exist yet) the device's free memory is the same before and
after it.

This file sorts last so that a run stopping at its first failure has already
run every other test.
"""
import numpy as np
import pytest

from forcesmith_b200 import synth
from forcesmith_b200.abi import FsError
from oracle import api as O
from tests.helpers import label, small_ternary, ternary_models, spline_pair_model

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def data():
    true, start = ternary_models(20)
    ds = label(small_ternary(6, 48, seed=99), true, O.Oracle, 1.0, 0.1)
    return ds, start


def _session(ds, model, precision):
    from forcesmith_b200.gpu import GpuSession
    g = GpuSession(0, precision)
    g.upload(ds)
    g.set_model(model)
    return g


def _noalloc(g, xs, w_e, w_s):
    import torch
    xs_t = torch.from_numpy(np.ascontiguousarray(xs, np.float64)).cuda()
    obj_t = torch.full((xs.shape[0],), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    g.eval_population_noalloc(xs_t.data_ptr(), xs.shape[0], obj_t.data_ptr(), w_e, w_s)
    torch.cuda.synchronize()  # the call runs on the context's stream
    return obj_t.cpu().numpy()


@pytest.mark.parametrize("precision,family", [("fp32", "eam"), ("fp64", "eam"), ("fp32", "pair")])
def test_noalloc_matches_population_twice(data, precision, family):
    ds, start = data
    model = start if family == "eam" else spline_pair_model(3, 14)
    g = _session(ds, model, precision)
    x0 = g.gather_params()
    for call, NP in enumerate((37, 20)):
        xs = np.stack([x0 * synth.uniform(x0.size, 0.97, 1.03, 1000 * call + k) for k in range(NP)])
        got = _noalloc(g, xs, 1.0, 0.1)
        want = g.eval_population(xs, 1.0, 0.1)
        assert np.all(np.isfinite(got))
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=0.0)


def test_noalloc_rejects_oversized_population(data):
    import torch
    ds, start = data
    g = _session(ds, start, "fp32")
    NP = 20000  # ≈ 4 KB of scratch per trial here, well past 8 MiB
    xs_t = torch.zeros((NP, g.D), dtype=torch.float64, device="cuda")
    obj_t = torch.zeros(NP, dtype=torch.float64, device="cuda")
    with pytest.raises(FsError) as e:
        g.eval_population_noalloc(xs_t.data_ptr(), NP, obj_t.data_ptr())
    assert "maximum" in str(e.value)


def test_noalloc_allocates_nothing(data):
    """Free device memory (cudaMemGetInfo) is unchanged across the first
    no-alloc call of a fresh context.  A first context runs the call once so
    that module loading and the address lookup are behind us."""
    import torch
    ds, start = data
    warm = _session(ds, start, "fp32")
    x0 = warm.gather_params()
    xs = np.stack([x0 * synth.uniform(x0.size, 0.97, 1.03, 77 + k) for k in range(16)])
    want = _noalloc(warm, xs, 1.0, 0.1)
    g = _session(ds, start, "fp32")
    xs_t = torch.from_numpy(xs).cuda()
    obj_t = torch.zeros(xs.shape[0], dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    g.eval_population_noalloc(xs_t.data_ptr(), xs.shape[0], obj_t.data_ptr(), 1.0, 0.1)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    np.testing.assert_allclose(obj_t.cpu().numpy(), want, rtol=1e-12, atol=0.0)


def test_noalloc_limit_in_message_is_exact(data):
    """The NP the refusal names is the largest that fits: it is accepted, and
    one more is refused."""
    import re
    import torch
    ds, start = data
    g = _session(ds, start, "fp32")
    NP = 20000
    xs_t = torch.zeros((NP + 1, g.D), dtype=torch.float64, device="cuda")
    obj_t = torch.zeros(NP + 1, dtype=torch.float64, device="cuda")
    with pytest.raises(FsError) as e:
        g.eval_population_noalloc(xs_t.data_ptr(), NP, obj_t.data_ptr())
    lim = int(re.search(r"NP <= (\d+)", str(e.value)).group(1))
    assert 0 < lim < NP
    xs_t[:lim] = torch.from_numpy(g.gather_params()).cuda()
    g.eval_population_noalloc(xs_t.data_ptr(), lim, obj_t.data_ptr())
    torch.cuda.synchronize()
    assert torch.isfinite(obj_t[:lim]).all()
    with pytest.raises(FsError):
        g.eval_population_noalloc(xs_t.data_ptr(), lim + 1, obj_t.data_ptr())
