"""Multi-rank host logic on CPU with the gloo backend (world size 2)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ddfacet_b200 import parallel


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = parallel.shard_facets(81, rank, world)
        # each rank "predicts" its facets: facet f contributes (f + 1) * (1 + 1j) to every vis
        pred = torch.zeros(16, dtype=torch.complex64)
        for f in mine:
            pred += (f + 1) * (1 + 1j)
        parallel.reduce_predictions(pred)
        t = parallel.max_over_ranks(10.0 + rank)
        q.put((rank, mine, pred.numpy().tolist(), t))
    finally:
        dist.destroy_process_group()


def test_facet_sharding_and_prediction_reduction_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    shards = [o[1] for o in out]
    assert sorted(sum(shards, [])) == list(range(81))
    assert abs(len(shards[0]) - len(shards[1])) <= 1
    want = sum(f + 1 for f in range(81))
    for o in out:
        assert all(abs(v - want * (1 + 1j)) < 1e-3 for v in o[2])
        assert o[3] == 11.0


@pytest.mark.parametrize("n,w", [(81, 8), (5, 8), (121, 3)])
def test_shard_facets_covers_all(n, w):
    got = [parallel.shard_facets(n, r, w) for r in range(w)]
    assert sorted(sum(got, [])) == list(range(n))


# ---- the composed sharded step, with stand-in degrid / grid calls (CPU tensors) ----

import dataclasses  # noqa: E402


@dataclasses.dataclass
class _Vis:
    vis: torch.Tensor


@dataclasses.dataclass
class _Facet:
    value: complex
    acc: torch.Tensor


def _fake_degrid(vs, facets, pol, jones, batch=None):
    """Subtracts each facet's "prediction" value * (1 + row index) from every visibility."""
    ramp = torch.arange(vs.vis.shape[0], dtype=torch.float32)[:, None] + 1
    for f in facets:
        vs.vis -= f.value * ramp


def _fake_grid(vs, facets, pol, jones, batch=None):
    """Adds the residuals, weighted by the facet's value, to each facet's accumulator."""
    for f in facets:
        f.acc += (vs.vis * f.value).sum(dim=0)


def _problem(nf=7):
    vis = torch.complex(torch.arange(40.0).reshape(10, 4), torch.ones(10, 4))
    model = [_Facet(complex(f + 1, -f), torch.zeros(4, dtype=torch.complex64)) for f in range(nf)]
    gridf = [_Facet(complex(1, f), torch.zeros(4, dtype=torch.complex64)) for f in range(nf)]
    return _Vis(vis.to(torch.complex64)), model, gridf


def _step_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        vs, model, gridf = _problem()
        mine = parallel.sharded_residual_step(vs, model, gridf, None, None, rank, world, degrid=_fake_degrid,
                                              grid=_fake_grid)
        q.put((rank, mine, vs.vis.numpy().tolist(), [gridf[i].acc.numpy().tolist() for i in mine]))
    finally:
        dist.destroy_process_group()


def test_sharded_residual_step_gloo():
    """Two ranks sharing a chunk: both end with the residuals of all facets' predictions, and each
    facet is gridded exactly once, with the same result as one rank doing every facet."""
    import numpy as np

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_step_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=120) for _ in range(world)])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    vs, model, gridf = _problem()
    mine = parallel.sharded_residual_step(vs, model, gridf, None, None, 0, 1, degrid=_fake_degrid, grid=_fake_grid)
    assert mine == list(range(len(model)))
    for o in out:
        np.testing.assert_allclose(np.array(o[2]), vs.vis.numpy(), rtol=1e-6)
    got = {f: acc for o in out for f, acc in zip(o[1], o[3])}
    assert sorted(got) == list(range(len(model)))
    for f, acc in got.items():
        np.testing.assert_allclose(np.array(acc), gridf[f].acc.numpy(), rtol=1e-5)
