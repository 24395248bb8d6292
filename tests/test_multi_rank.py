"""Multi-GPU host logic on CPU: two gloo ranks.

The path shards at case granularity with no exchange on the data path: under torchrun each rank
runs its own replica of the workload (seeds shifted by the rank), and the reported time of a
step is the max over ranks.  These tests run the same helpers bench.py uses, on two processes
with the gloo backend (no GPU).
"""
import os
import socket

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    import sys
    import datetime
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import __graft_entry__ as entry
        pkg = entry.load_package()
        items, kind = bench.build_workload(pkg, "ws-153", "fast", seed_offset=bench.replica_seed_offset(rank))
        sig = np.array([[p.imax, p.jmax, p.Re, p.Da, p.InvFr2] for p, *_ in items], np.float64)
        # every rank sees every rank's case table
        t = torch.from_numpy(sig.ravel().copy())
        gathered = [torch.zeros_like(t) for _ in range(world)]
        dist.all_gather(gathered, t)
        # max over ranks of a rank-dependent elapsed time
        elapsed = 1.0 + 0.5 * rank
        mx = bench.max_over_ranks(elapsed, world)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), tables=np.stack([g.numpy() for g in gathered]),
                 max=mx, kind=kind, n=len(items))
    finally:
        dist.destroy_process_group()


def test_replicas_and_max_over_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    for r in res:
        assert float(r["max"]) == 1.5            # the slowest rank's time
        assert int(r["n"]) == 64 and str(r["kind"]) == "full"
    tables = res[0]["tables"].reshape(world, 64, 5)
    assert np.array_equal(res[0]["tables"], res[1]["tables"])   # both ranks agree on the plan
    # same case sizes on every rank (weak scaling), different cases (parameters differ)
    assert np.array_equal(tables[0][:, :2], tables[1][:, :2])
    assert not np.array_equal(tables[0][:, 2:], tables[1][:, 2:])


def test_single_rank_is_identity():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, 1) == 3.25
    assert bench.replica_seed_offset(0) == 0
