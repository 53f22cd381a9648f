"""Windows split across ranks (CPU, two gloo ranks): every window in exactly one share, and the
windows of both ranks, gathered, give the same combined models as one rank running them all.

The time-lapse windows are independent (adtlert/inversion/core.py:445-577 inverts each from its
own initial models), so ``bench.py --gpus N --workload timelapse`` gives each rank the share
``window_share`` returns and needs no collective on the data path. Here each rank inverts its share
with the FP64 oracle driver on a small series; rank 0 gathers."""

import multiprocessing as mp
import os
import socket
import sys

import numpy as np

from adtlert_b200.timelapse import window_share, window_starts
from conftest import ROOT


def test_shares_partition_the_windows():
    for count in (0, 1, 5, 363):
        for world in (1, 2, 3, 8):
            shares = [window_share(count, r, world) for r in range(world)]
            assert sorted(i for s in shares for i in s) == list(range(count))
            assert max(map(len, shares)) - min(map(len, shares)) <= 1


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _inputs():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    golden = np.load(ROOT / "tests" / "golden" / "timelapse_small.npz")
    return golden["observed_log"], golden["initial_log"], golden["settings"]


def _window_models(share):
    from cases import case_inputs
    from oracle.timelapse import OracleTimeLapse

    observed, initial, settings = _inputs()
    inputs = case_inputs("tri_flat")
    oracle = OracleTimeLapse(inputs["nodes"], inputs["cells"], inputs["electrodes"], inputs["measurements"],
                             max_iterations=2, data_std=float(settings[1]))
    starts = window_starts(observed.shape[0], 3)
    return {i: oracle.invert_window(observed[starts[i]:starts[i] + 3], initial[starts[i]:starts[i] + 3])[0]
            for i in share}


def _rank(rank: int, port: int, queue) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                      CUDA_VISIBLE_DEVICES="")
    sys.path[:0] = [str(ROOT), str(ROOT / "ad-tlert_b200")]
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=2)
    observed, _, _ = _inputs()
    share = window_share(len(window_starts(observed.shape[0], 3)), rank, 2)
    gathered = [None, None]
    dist.all_gather_object(gathered, _window_models(share))
    if rank == 0:
        queue.put({i: m for part in gathered for i, m in part.items()})
    dist.destroy_process_group()


def test_two_ranks_give_the_one_rank_result():
    ctx = mp.get_context("spawn")
    queue, port = ctx.Queue(), _free_port()
    ranks = [ctx.Process(target=_rank, args=(r, port, queue)) for r in range(2)]
    for p in ranks:
        p.start()
    models = queue.get(timeout=300)
    for p in ranks:
        p.join(timeout=60)
        assert p.exitcode == 0
    observed, _, _ = _inputs()
    count = len(window_starts(observed.shape[0], 3))
    assert sorted(models) == list(range(count))  # no window dropped or duplicated
    single = _window_models(range(count))
    for i in range(count):
        assert np.array_equal(models[i], single[i])
