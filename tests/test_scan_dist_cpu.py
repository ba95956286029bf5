"""Replica split of the batched scan on CPU: two gloo ranks, a stand-in runner
in place of the GPU solves; every case is solved by exactly one rank and the
gathered results come back in case order."""

import os
import socket
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_runner(cases, **_kw):
    hists = [dict(best_sigma=0.1 * c["id"], best_iter=c["id"], sigma=[1.0] * (c["id"] + 1),
                  stop_reason="sigma_stall") for c in cases]
    cells = sum(c["id"] + 1 for c in cases)
    return hists, dict(setup_s=0.5, scan_s=1.0 + len(cases), cell_iterations=cells, gcell_iter_per_s=0.0)


def _rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import json

    import torch.distributed as dist

    from nfgs_b200 import scan

    dist.init_process_group("gloo", rank=rank, world_size=world)
    cases = [dict(id=i) for i in range(7)]
    results, timing = scan.distributed_scan(cases, dist, rank, world, runner=_fake_runner)
    dist.destroy_process_group()
    Path(out_dir, f"r{rank}.json").write_text(json.dumps(dict(results=results, timing=timing)))


def test_shard_cases():
    from nfgs_b200.scan import shard_cases

    cases = list(range(10))
    parts = [shard_cases(cases, r, 3) for r in range(3)]
    assert sorted(i for p in parts for i in p) == cases
    assert parts[0] == [0, 3, 6, 9]


def test_two_rank_scan(tmp_path):
    import json

    import torch.multiprocessing as mp

    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(2):
        d = json.loads((tmp_path / f"r{r}.json").read_text())
        assert [x["best_iter"] for x in d["results"]] == list(range(7))
        assert [x["iterations"] for x in d["results"]] == [i + 1 for i in range(7)]
        t = d["timing"]
        assert t["ranks"] == 2 and t["cell_iterations"] == sum(i + 1 for i in range(7))
        assert t["scan_s"] == 5.0  # the slower rank: 4 cases
