"""The N > 1 host logic of bench.py on CPU: two gloo ranks (the path runs
independent replicas; the only exchanges are the barrier and the max over
ranks of the timed region), and the reference arm's rank-0-only rule."""

import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench

    w, r, local, pg = bench.dist_setup()
    assert (w, r) == (world, rank) and pg is not None
    bench.barrier_sync(pg, local)
    got = bench.max_over_ranks(pg, 1.5 * (rank + 1), local)
    # the reference arm: rank 0 alone runs; the others return 0 without work
    other = bench.run_reference(None) if rank != 0 else 0
    pg.barrier()
    pg.destroy_process_group()
    Path(out_dir, f"rank{rank}.txt").write_text(f"{got} {other}")


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    for r in range(world):
        got, other = (tmp_path / f"rank{r}.txt").read_text().split()
        assert float(got) == 3.0
        assert int(other) == 0
