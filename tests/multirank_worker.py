"""Worker of the two-rank CPU test (tests/test_multirank.py): one gloo rank
running the host logic of bench.py's multi-rank ensemble path."""
import datetime
import importlib.util
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("dcm_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def worker(rank, world, port, queue):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench = load_bench()
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from conftest import load_dcm
        load_dcm()
        from dcm_b200 import cases
        spec = cases.ensemble_members(64)
        mine = bench.partition(spec, rank, world)
        R = bench.Ranks(dist)
        pts = sum(ip * jp * kp for ip, jp, kp, _, _ in mine)
        total = R.sum(pts)
        longest = R.max(1.5 * (rank + 1))  # a per-rank time: the job takes the slowest
        R.barrier()
        queue.put((rank, [m[4] for m in mine], pts, total, longest,
                   sum(ip * jp * kp for ip, jp, kp, _, _ in spec)))
    finally:
        dist.destroy_process_group()
