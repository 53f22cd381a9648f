"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (the GPU runs use NCCL the same way).

Each rank of ``bench.py --gpus N`` times its own models; the job time is the maximum over ranks
(``max_over_ranks``) between barriers, and the reference arm runs on rank 0 alone."""

import multiprocessing as mp
import os
import socket
import sys

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, port: int, queue) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                      LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench

    got_rank, world = bench.dist_setup(None)
    bench.barrier(world)
    slowest = bench.max_over_ranks(1.5 * (rank + 1), world)
    bench.barrier(world)
    queue.put((got_rank, world, slowest, dist.get_backend()))
    dist.destroy_process_group()


def test_two_gloo_ranks_time_the_job_as_the_slowest_rank():
    ctx = mp.get_context("spawn")
    queue, port = ctx.Queue(), _free_port()
    ranks = [ctx.Process(target=_rank, args=(r, port, queue)) for r in range(2)]
    for p in ranks:
        p.start()
    results = sorted(queue.get(timeout=120) for _ in ranks)
    for p in ranks:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results == [(0, 2, 3.0, "gloo"), (1, 2, 3.0, "gloo")]


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    calls = []
    monkeypatch.setattr(bench, "run_reference", lambda args, rank, world: calls.append((rank, world)) or {"impl": "reference"})
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference"])
    for rank in ("1", "0"):
        monkeypatch.setenv("RANK", rank)
        monkeypatch.setenv("WORLD_SIZE", "2")
        bench.main()
    assert calls == [(0, 2)]
    assert capsys.readouterr().out.strip() == '{"impl": "reference"}'
