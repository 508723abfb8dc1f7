"""Scenes across GPUs (natray_b200.replicas), the host side, on the CPU: the request stream
shared out by free device memory, the ranks' results merged, and the two-rank path through
torch.distributed with the gloo backend (world size 2, one process per rank)."""
import json
import socket
import sys
from pathlib import Path

import numpy as np

from natray_b200 import Params, build_world
from natray_b200.replicas import device_bytes, merge_results, partition_requests


def test_partition_is_least_loaded_first():
    # rank 0 has 10 units free, rank 1 has 7: the 4-unit requests alternate as the free memory
    # left says, ties to the lower rank
    plan = partition_requests([4, 4, 4, 4, 1], [10, 7])
    assert plan == [[0, 2, 4], [1, 3]]  # left: 10,7 -> 6,7 -> 6,3 -> 2,3 -> 2,-1 -> 1,-1
    assert partition_requests([5, 5, 5], [0, 0]) == [[0, 2], [1]]  # nothing fits: still least loaded
    p = partition_requests([1] * 6, [3, 3, 3])
    assert sorted(sum(p, [])) == list(range(6)) and [len(x) for x in p] == [2, 2, 2]


def test_merge_results():
    a = {"requests": 2, "seconds": 1.0, "latencies": [0.1, 0.3]}
    b = {"requests": 3, "seconds": 2.0, "latencies": [0.2, 0.4, 0.5]}
    m = merge_results([a, b])
    assert m["requests"] == 5 and m["seconds"] == 2.0 and m["scenes_per_s"] == 2.5 and m["per_rank"] == [2, 3]
    assert np.isclose(m["p50_s"], 0.3) and np.isclose(m["p99_s"], np.percentile([0.1, 0.2, 0.3, 0.4, 0.5], 99))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_over_gloo(tmp_path):
    import torch.multiprocessing as mp
    sys.path.insert(0, str(Path(__file__).parent))
    import replica_worker

    worlds = [build_world(Params(resolution=r, mesh_level=2, block_cap=b)) for r, b in
              [(12, 512), (12, 2048), (14, 512), (12, 1024), (14, 4096)]]
    blobs = [bytes(w.blob) for w in worlds]
    arrivals = [0.0, 0.01, 0.02, 0.03, 0.04]
    frees = [300_000_000, 200_000_000]  # about three and two of these scenes
    mp.spawn(replica_worker.run, args=(free_port(), blobs, arrivals, frees, str(tmp_path)), nprocs=2, join=True)
    r0 = json.loads((tmp_path / "rank0.json").read_text())
    r1 = json.loads((tmp_path / "rank1.json").read_text())
    assert r1["merged"] is None and r0["max"] == r1["max"] == 2.5
    m = r0["merged"]
    want = partition_requests([device_bytes(w) for w in worlds], frees)
    assert m["plan"] == want and m["requests"] == 5 and m["per_rank"] == [len(x) for x in want]
    assert m["p50_s"] == 0.01 and m["p99_s"] == 0.01
    assert len(want[0]) > len(want[1]) > 0  # the rank with more memory takes more
