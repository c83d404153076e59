"""One field over several ranks (asz_compress_slab).

CPU: the slab layout covers every axis-0 plane once, with each slab's lower face owned by the slab
below; the torch.distributed callbacks (world size 2 over gloo) reduce, gather and pass bytes as the
library expects.
GPU: 2 or 3 processes, each with its own context on device 0 and a slab of the field, exchange over
gloo; rank 0's .asz must equal asz_compress on the whole field byte for byte. The processes'
kernels never wait on one another: every exchange goes through the host.
"""
import os
import socket
import sys
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT

CASES = [
    # shape, plan, family, rel_eb, block_pivot_ratio, ranks
    ((48, 40, 36), "cubic0_012,cubic1_012,cubic2_012,cubic0_012,cubic1_012,cubic2_012", "cubic", 1e-3, 3, 2),
    ((48, 40, 36), "cubic0_012,cubic1_012,cubic2_012,cubic0_012,cubic1_012,cubic2_012", "quintic", 1e-3, 3, 2),
    ((64, 24, 40), "cubic0_120,cubic0_021,cubic1_012,cubic2_012,cubic0_012", "quintic", 1e-2, 2, 3),
    ((40, 30, 50), "cubic2_012,cubic2_012,cubic2_012,cubic2_012", "cubic", 1e-3, 3, 2),
    ((30, 20, 20), "cubic0_012,cubic1_012,cubic2_012", "cubic", 1e-4, 1, 3),
]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _field(shape, seed):
    from asz_b200 import fields
    return fields.c2_field(seed=seed, shape=shape)


def test_layout_covers_every_plane_once():
    from asz_b200 import api, slabs
    for shape, plan, _, _, bpr, _ in CASES:
        p = api.default_params(block_pivot_ratio=bpr)
        nb = slabs.blocks_of(shape, plan, p)
        for world in range(1, min(nb, 5) + 1):
            seen = []
            for b0, b1 in slabs.split_blocks(nb, world):
                pb, pc, nb2 = slabs.slab_planes(shape, plan, b0, b1, p)
                assert nb2 == nb and pc > 0
                seen.extend(range(pb, pb + pc))
            assert seen == list(range(shape[0]))
    with pytest.raises(api.AszError):
        slabs.slab_planes((40, 20, 30), "cubic0_012", 3, 3)
    with pytest.raises(api.AszError):
        slabs.slab_planes((40, 20, 30), "cubic0_012", 0, 99)
    with pytest.raises(ValueError):
        slabs.split_blocks(2, 3)


def _comm_worker(rank, world, port, outdir):
    sys.path.insert(0, ROOT)
    import ctypes as C
    import datetime

    import torch.distributed as dist

    from asz_b200 import slabs
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    cm = slabs.TorchComm(dist)
    s = cm.struct
    res = []
    f = np.array([1.5 + rank, -2.0 * rank], np.float32)
    assert s.allreduce(None, f.ctypes.data, 2, 0, 0) == 0
    res.append(f.tolist())
    u = np.array([10 + rank, 2 ** 40], np.uint64)
    assert s.allreduce(None, u.ctypes.data, 2, 1, 0) == 0
    res.append([int(v) for v in u])
    i = np.array([rank - 5, rank + 7], np.int32)
    assert s.allreduce(None, i.ctypes.data, 2, 2, 1) == 0
    res.append(i.tolist())
    j = np.array([rank - 5, rank + 7], np.int32)
    assert s.allreduce(None, j.ctypes.data, 2, 2, 2) == 0
    res.append(j.tolist())
    mine = np.arange(5, dtype=np.uint8) + 10 * rank
    got = np.zeros(5 * world, np.uint8)
    assert s.allgather(None, mine.ctypes.data, 5, got.ctypes.data) == 0
    res.append(got.tolist())
    if rank == 0:
        msg = np.arange(7, dtype=np.uint8) * 3
        assert s.send(None, msg.ctypes.data, 7, 1) == 0
    else:
        buf = np.zeros(7, np.uint8)
        assert s.recv(None, buf.ctypes.data, 7, 0) == 0
        res.append(buf.tolist())
    with open(os.path.join(outdir, f"r{rank}.txt"), "w") as fh:
        fh.write(repr(res))
    dist.barrier()
    dist.destroy_process_group()


def test_torch_comm_callbacks_over_gloo():
    port = _free_port()
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_comm_worker, args=(2, port, d), nprocs=2, join=True, start_method="spawn")
        r0 = eval(open(os.path.join(d, "r0.txt")).read())
        r1 = eval(open(os.path.join(d, "r1.txt")).read())
    for r in (r0, r1):
        assert r[0] == [4.0, -2.0]
        assert r[1] == [21, 2 ** 41]
        assert r[2] == [-5, 7]
        assert r[3] == [-4, 8]
        assert r[4] == [0, 1, 2, 3, 4, 10, 11, 12, 13, 14]
    assert r1[5] == [0, 3, 6, 9, 12, 15, 18]


def _slab_worker(rank, world, port, outdir, case_index):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    from asz_b200 import api, slabs
    shape, plan, family, rel_eb, bpr, _ = CASES[case_index]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    x = _field(shape, 30 + case_index)
    p = api.default_params(block_pivot_ratio=bpr)
    nb = slabs.blocks_of(shape, plan, p)
    b0, b1 = slabs.split_blocks(nb, world)[rank]
    pb, pc, _ = slabs.slab_planes(shape, plan, b0, b1, p)
    with api.Context(0) as ctx:
        blob, rep = slabs.compress_slab(ctx, slabs.TorchComm(dist), x[pb:pb + pc], shape, b0, b1, rel_eb, plan, family,
                                        api.default_params(block_pivot_ratio=bpr))
        if rank == 0:
            whole, wrep = ctx.compress(x, rel_eb, plan, family, api.default_params(block_pivot_ratio=bpr))
            with open(os.path.join(outdir, "slab.asz"), "wb") as f:
                f.write(blob)
            with open(os.path.join(outdir, "whole.asz"), "wb") as f:
                f.write(whole)
            with open(os.path.join(outdir, "rep.txt"), "w") as f:
                f.write(f"{rep.asz_len} {rep.pre_zstd_len} {rep.default_slope!r} {wrep.default_slope!r} "
                        f"{rep.min_val!r} {rep.max_val!r} {rep.reruns}\n")
        else:
            assert blob is None
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("case_index", range(len(CASES)))
def test_slab_compression_equals_whole_field(case_index):
    world = CASES[case_index][5]
    port = _free_port()
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_slab_worker, args=(world, port, d, case_index), nprocs=world, join=True,
                           start_method="spawn")
        slab = open(os.path.join(d, "slab.asz"), "rb").read()
        whole = open(os.path.join(d, "whole.asz"), "rb").read()
        rep = open(os.path.join(d, "rep.txt")).read().split()
    assert int(rep[0]) == len(slab)
    assert rep[2] == rep[3], "default slope differs from the whole field's"
    assert slab == whole, ".asz of the slabs differs from the whole-field compression"


def _fullsize_worker(rank, world, port, outdir):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import datetime
    import hashlib

    import torch.distributed as dist

    import make_fullsize
    from asz_b200 import api, slabs
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=300))
    x = make_fullsize.make_field("c2")
    plan = ",".join(["cubic2_012"] * 9)
    p = api.default_params(block_pivot_ratio=3)
    b0, b1 = slabs.split_blocks(slabs.blocks_of(x.shape, plan, p), world)[rank]
    pb, pc, _ = slabs.slab_planes(x.shape, plan, b0, b1, p)
    with api.Context(0) as ctx:
        blob, _ = slabs.compress_slab(ctx, slabs.TorchComm(dist), x[pb:pb + pc], x.shape, b0, b1, 1e-3, plan, "cubic",
                                      api.default_params(block_pivot_ratio=3))
    if rank == 0:
        with open(os.path.join(outdir, "digest.txt"), "w") as f:
            f.write(hashlib.sha256(x.tobytes()).hexdigest() + " " + hashlib.sha256(blob).hexdigest() + "\n")
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.gpu
def test_slabs_at_full_size_match_the_reference_record():
    """The 512^3 C2 field at REL 1e-3 (cubic2_012 x9, block pivot ratio 3) over 2 ranks: rank 0's
    .asz has the digest the reference binaries' output has (tests/golden/fullsize.json)."""
    import json
    fix = json.load(open(os.path.join(ROOT, "tests", "golden", "fullsize.json")))
    case = next(c for c in fix["cases"] if c["name"] == "c2_cubic_0.001")
    port = _free_port()
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_fullsize_worker, args=(2, port, d), nprocs=2, join=True, start_method="spawn")
        field_sha, asz_sha = open(os.path.join(d, "digest.txt")).read().split()
    if field_sha != fix["fields"]["c2"]["sha256"]:
        pytest.skip("generated input differs from the recorded one (other NumPy build)")
    assert asz_sha == case["asz_sha256"]
