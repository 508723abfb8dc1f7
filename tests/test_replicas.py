"""Scenes across GPUs (natray_b200.replicas), the host side, on the CPU: the request dispatch as
slots free up (a claim counter every server shares), the ranks' results merged, and the two-rank
path through torch.distributed with the gloo backend (world size 2, one process per rank)."""
import json
import socket
import sys
from pathlib import Path

import numpy as np

from natray_b200.replicas import merge_results
from natray_b200.serve import LocalRequests, SharedRequests


class DictStore:
    """The add() of a torch.distributed store, in one process."""

    def __init__(self):
        self.v = {}

    def add(self, key, n):
        self.v[key] = self.v.get(key, 0) + n
        return self.v[key]


def test_local_requests_come_in_arrival_order():
    r = LocalRequests([0.0, 0.5, 1.0])
    assert r.claim(0.1) == 0 and r.claim(0.1) is None and r.wait_hint(0.1) == 0.4
    assert r.claim(1.0) == 1 and r.claim(1.0) == 2 and r.exhausted()


def test_shared_requests_go_to_one_server_each():
    store = DictStore()
    arr = [0.0, 0.0, 0.2, 0.3]
    a, b = SharedRequests(store, arr), SharedRequests(store, arr)
    got = [a.claim(0.0), b.claim(0.0), a.claim(0.0), b.claim(0.0)]
    assert got[:2] == [0, 1] and got[2:] == [None, None]  # 2 and 3 are claimed but not arrived
    assert a.wait_hint(0.0) == 0.2 and b.wait_hint(0.0) == 0.3
    assert a.claim(0.25) == 2 and b.claim(0.25) is None and b.claim(0.3) == 3
    assert a.claim(1.0) is None and b.claim(1.0) is None and a.exhausted() and b.exhausted()


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
    # 40 requests arriving over 0.2 s, 2 slots a rank, rank 1's steps four times slower: every
    # request is served exactly once, by the rank that had room first, so rank 1 serves fewer.
    import torch.multiprocessing as mp
    sys.path.insert(0, str(Path(__file__).parent))
    import replica_worker

    n = 40
    arrivals = [0.005 * i for i in range(n)]
    port = free_port()
    mp.spawn(replica_worker.run, args=(port, n, arrivals, [2.0, 8.0], 2, str(tmp_path)), nprocs=2, join=True)
    r0 = json.loads((tmp_path / "rank0.json").read_text())
    r1 = json.loads((tmp_path / "rank1.json").read_text())
    assert r1["merged"] is None and r0["max"] == r1["max"] == 2.5
    m = r0["merged"]
    a, b = m["served_by_rank"]
    assert sorted(a + b) == list(range(n)) and not set(a) & set(b)
    assert m["requests"] == n and m["per_rank"] == [len(a), len(b)]
    assert len(a) > len(b) > 0
    assert m["p50_s"] > 0 and m["p99_s"] >= m["p50_s"]
