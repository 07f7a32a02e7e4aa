"""Multi-process host logic of chfem_b200.distributed on the CPU: world size 2 over gloo
(127.0.0.1), one process per rank, the GPU solve replaced by a CPU function."""
import os
import socket
import sys

import pytest

from tests import helpers as H


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, out_dir):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, H.ROOT)
    from chfem_b200 import distributed as D
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    try:
        if mode == "map":
            items = list(range(11))
            res = D.map_samples(lambda chunk: [v * v + rank * 0 for v in chunk], items)
            t = D.max_over_ranks(1.5 + rank)
            with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
                f.write(f"{res}\n{t}\n")
        elif mode == "fail":
            # rank 1 fails inside its shard; the error surfaces on that rank
            def fn(chunk):
                if rank == 1:
                    raise ValueError("solver failed on rank 1")
                return chunk
            try:
                D.map_samples(fn, list(range(4)))
            except ValueError as e:
                with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
                    f.write(str(e))
                raise
    finally:
        if mode == "map":
            dist.destroy_process_group()


def _spawn(mode, tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.start_processes(_worker, args=(2, port, mode, str(tmp_path)), nprocs=2, join=False, start_method="spawn")
    return ctx


def test_map_samples_gathers_in_order(tmp_path):
    ctx = _spawn("map", tmp_path)
    while not ctx.join(timeout=60):
        pass
    for rank in range(2):
        lines = open(tmp_path / f"r{rank}.txt").read().split("\n")
        assert lines[0] == str([v * v for v in range(11)])
        assert float(lines[1]) == 2.5


def test_rank_failure_surfaces(tmp_path):
    """A rank whose solve raises ends with that error; the other rank does not hang past the
    process-group timeout."""
    ctx = _spawn("fail", tmp_path)
    with pytest.raises(Exception):
        while not ctx.join(timeout=90):
            pass
    assert "solver failed on rank 1" in open(tmp_path / "r1.txt").read()


def test_shard_range_partitions():
    from chfem_b200.distributed import shard_range
    for n in range(0, 30):
        for world in range(1, 7):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            assert max(h - l for l, h in spans) - min(h - l for l, h in spans) <= 1
    with pytest.raises(ValueError):
        shard_range(3, 2, 2)
