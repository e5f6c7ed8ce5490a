"""The multi-rank path on CPU: world size 2 over gloo.  Each rank evaluates
the normal equations of its shard of the configurations (with the oracle as
the evaluator, since this runs without a GPU), the ranks sum them with one
all-reduce, and the result must equal the single-process evaluation of all
configurations (relative 1e-10: only the summation order differs)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from forcesmith_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problem():
    from oracle import api as O
    from tests.helpers import label, small_ternary, ternary_models
    true, start = ternary_models(8)
    ds = small_ternary(5, 32, seed=17)
    ds = label(ds, true, O.Oracle, 1.0, 0.1)
    return ds, start


def _normal_equations(ds, model):
    from oracle import api as O
    o = O.Oracle()
    o.upload(ds)
    o.set_model(model)
    F = o.eval(1.0, 0.1, want=("F",))["F"]
    J = o.jacobian_analytic(1.0, 0.1)
    JtJ, Jtr = O.normal_equations(J, F)
    return JtJ, Jtr, float(F @ F)


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ds, start = _problem()
        mine = shard.shard_configs(ds.natoms, world)[rank]
        JtJ, Jtr, obj = _normal_equations(ds.subset(mine), start)
        JtJ, Jtr, obj = shard.allreduce_normal_equations(JtJ, Jtr, obj)
        out[rank] = (JtJ, Jtr, obj)
    finally:
        dist.destroy_process_group()


def test_shards_cover_every_configuration_once():
    natoms = np.array([64, 512, 216, 216, 64, 512, 32, 300])
    parts = shard.shard_configs(natoms, 3)
    allc = np.sort(np.concatenate(parts))
    assert np.array_equal(allc, np.arange(natoms.size))
    loads = [natoms[p].sum() for p in parts]
    assert max(loads) - min(loads) <= natoms.max()
    assert [list(p) for p in parts] == [list(p) for p in shard.shard_configs(natoms, 3)]


def test_pack_roundtrip():
    D = 5
    A, b = np.arange(D * D, dtype=float).reshape(D, D), np.arange(D, dtype=float)
    A2, b2, o2 = shard.unpack_normal_equations(shard.pack_normal_equations(A, b, 3.5), D)
    assert np.array_equal(A, A2) and np.array_equal(b, b2) and o2 == 3.5


def test_two_ranks_sum_to_the_whole():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=240)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    ds, start = _problem()
    JtJ, Jtr, obj = _normal_equations(ds, start)
    for r in range(world):
        A, b, o = res[r]
        np.testing.assert_allclose(A, JtJ, rtol=1e-10, atol=1e-12 * np.abs(JtJ).max())
        np.testing.assert_allclose(b, Jtr, rtol=1e-10, atol=1e-12 * np.abs(Jtr).max())
        assert o == pytest.approx(obj, rel=1e-12)
