"""Multi-rank path of bench.py on CPU: two gloo ranks build independent replica problems
(seeded per rank, same size) and reduce their times with max; no GPU involved."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    from bem_for_nonlinear_waves_b200.bvp import inspect_plan
    cfg = dict(bench.CONFIGS["tank_2800"])
    cfg["tank"] = dict(cfg["tank"], h=0.125, noise=0.2)
    t, d, kv = bench.make_problem(cfg, rank)
    _, _, st = inspect_plan(t.X, t.tri, t.face_dirichlet, d, expansion_order=cfg["p"])
    mine = float(rank + 1) * 0.5
    mx = bench.allreduce_max([mine, float(st["nnz"])], world, device="cpu")
    out[rank] = (float(t.X[:, 2].max()), st["nnz"], mx[0], mx[1])
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        r = dict(out)
    assert set(r) == {0, 1}
    # independent seeded replicas: different free-surface noise
    assert r[0][0] != r[1][0]
    # max over ranks is seen identically by both ranks
    assert r[0][2] == r[1][2] == 1.0
    assert r[0][3] == r[1][3] == max(r[0][1], r[1][1])
