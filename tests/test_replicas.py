"""Multi-GPU replicas on CPU: world size 2 over gloo. Each rank compresses its share of the fields
(here with the CPU oracle, the reference's algorithm) and the slowest rank's time and the total
bytes are reduced; every field is compressed exactly once, and each matches a single-process run."""
import os
import socket
import sys
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from asz_b200.replicas import assign

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
SHAPES = [(12, 14, 16), (9, 20, 11), (16, 16, 16), (7, 8, 30), (21, 10, 10)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _field(i):
    rng = np.random.default_rng(100 + i)
    from asz_b200 import fields
    return fields.grf_field(SHAPES[i], 3.0, rng).astype(np.float32)


def _worker(rank, world, port, outdir):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch.distributed as dist

    import oracle as O
    from asz_b200 import replicas
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sizes = [4 * int(np.prod(s)) for s in SHAPES]

    def fn(i):
        c = O.compress(_field(i), 1e-3, "cubic0_012,cubic1_012,cubic2_012", False, O.default_params(block_pivot_ratio=2))
        return c.asz

    r = replicas.run(sizes, fn, dist=dist)
    for u, blob in zip(r.units, r.results):
        with open(os.path.join(outdir, f"{u}.asz"), "wb") as f:
            f.write(blob)
    with open(os.path.join(outdir, f"rank{rank}.txt"), "w") as f:
        f.write(f"{r.max_s} {r.local_s} {r.total_bytes} {' '.join(map(str, r.units))}\n")
    dist.barrier()
    dist.destroy_process_group()


def test_assign_balances_and_covers():
    sizes = [100, 90, 80, 10, 10, 5, 1]
    parts = assign(sizes, 3)
    flat = sorted(u for p in parts for u in p)
    assert flat == list(range(len(sizes)))
    loads = [sum(sizes[u] for u in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes)
    assert assign(sizes, 3) == parts  # deterministic


def test_two_rank_replicas_over_gloo():
    import oracle as O
    port = _free_port()
    with tempfile.TemporaryDirectory() as outdir:
        mp.start_processes(_worker, args=(2, port, outdir), nprocs=2, join=True, start_method="spawn")
        lines = [open(os.path.join(outdir, f"rank{r}.txt")).read().split() for r in range(2)]
        max_s = [float(l[0]) for l in lines]
        local_s = [float(l[1]) for l in lines]
        total = [int(l[2]) for l in lines]
        units = sorted(int(u) for l in lines for u in l[3:])
        assert units == list(range(len(SHAPES)))  # every field exactly once
        assert max_s[0] == max_s[1] == pytest.approx(max(local_s))
        assert total[0] == total[1] == sum(4 * int(np.prod(s)) for s in SHAPES)
        for i in range(len(SHAPES)):
            want = O.compress(_field(i), 1e-3, "cubic0_012,cubic1_012,cubic2_012", False,
                              O.default_params(block_pivot_ratio=2)).asz
            assert open(os.path.join(outdir, f"{i}.asz"), "rb").read() == want
