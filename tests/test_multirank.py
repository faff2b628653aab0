"""The bench's multi-rank path on CPU (gloo, world_size 2): replicas solve
different seeded systems and every timing is the maximum over ranks."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, ws, port, out):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        got_ws, got_rank, _ = bench.dist_init()
        out[rank] = (got_ws, got_rank, bench.max_over_ranks(1.5 + rank, ws), bench.rank_seed(rank))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_seeds_with_gloo():
    ws = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(ws, _free_port(), out), nprocs=ws, join=True)
        res = dict(out)
    assert res[0][:3] == (2, 0, 2.5) and res[1][:3] == (2, 1, 2.5)
    assert res[0][3] != res[1][3]
