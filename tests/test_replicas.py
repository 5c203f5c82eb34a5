"""Multi-GPU runs are replicas (one process per GPU, queries sharded, no
collective on the data path).  The measurement plumbing (rover_b200.replicas)
runs here on two CPU processes over gloo: max-over-ranks timing, rank 0's
picked configuration shared with every rank, a decision all ranks take
together, whole-job throughput."""
from __future__ import annotations

import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    import json

    import torch

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from rover_b200 import replicas
    dist = replicas.init("gloo", timeout_s=60)
    dev = torch.device("cpu")
    res = {
        # rank r timed 10 * r + 1 ms: the job took the slowest rank's time
        "max_ms": replicas.max_over_ranks(dist, 10.0 * rank + 1.0, dev),
        # only rank 0 reached the target: nobody times the gated form
        "all_ok": replicas.all_ranks(dist, rank == 0, dev),
        "all_ok_true": replicas.all_ranks(dist, True, dev),
        # each rank calibrated its own point; rank 0's is timed everywhere
        "pick": replicas.from_rank0(dist, {"L": 64 if rank == 0 else 32, "stop": float("inf")}),
    }
    res["qps"] = replicas.throughput(10000, 5, world, res["max_ms"])
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def test_replica_plumbing_two_gloo_ranks(tmp_path):
    torch = pytest.importorskip("torch")
    import json

    import torch.multiprocessing as mp
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
        assert p.exitcode == 0
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for r in res:
        assert r["max_ms"] == 11.0
        assert r["all_ok"] is False and r["all_ok_true"] is True
        assert r["pick"]["L"] == 64 and r["pick"]["stop"] == float("inf")
        assert abs(r["qps"] - 10000 * 5 * 2 / 0.011) < 1e-6 * r["qps"]
