"""The multi-GPU host logic of bench.py on CPU: two gloo ranks (world size 2) take the
max over ranks of their device times, as the replicas run does over NCCL."""
import os
import socket
import sys

import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = [3.25, 7.5][rank]
        got = bench.max_over_ranks(dist, local_ms, device="cpu")
        with open(os.path.join(out_dir, "rank%d" % rank), "w") as f:
            f.write(repr(got))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks(tmp_path):
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        assert float((tmp_path / ("rank%d" % r)).read_text()) == 7.5


def test_max_over_ranks_without_a_process_group():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks(None, 4.0) == 4.0
