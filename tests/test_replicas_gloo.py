"""The N-GPU path of bench.py is replicas only: every rank runs its own copy
of the batch and only timing values cross ranks (a MAX for the step time, a
SUM for counts), over gloo.  Two ranks on CPU check that plumbing: the
reduction results, the barrier, and the whole-job value formula
(world x instances x steps / max time)."""
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist()
    local_ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
    d.barrier()
    ms = d.max(local_ms)
    total = d.sum(float(rank + 1))
    value = d.world * 64 * 3 / (ms / 1e3)
    with open(os.path.join(outdir, f"r{rank}.json"), "w") as f:
        json.dump({"world": d.world, "rank": d.rank, "ms": ms, "sum": total, "value": value}, f)
    d.close()


@pytest.mark.timeout(180)
def test_two_gloo_ranks(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    rows = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    for r in rows:
        assert r["world"] == 2
        assert r["ms"] == 150.0           # MAX over ranks
        assert r["sum"] == 3.0            # SUM over ranks
        assert abs(r["value"] - 2 * 64 * 3 / 0.150) < 1e-9
