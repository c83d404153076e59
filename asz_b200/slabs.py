"""One field compressed by several ranks, each holding a slab of axis-0 planes (asz_compress_slab).

The reference compresses a field block by block in raster order (c_codes/asz_core/compress.tpp:
179-209). A slab is a run of axis-0 blocks; its blocks are contiguous in every stream of the .asz,
so the ranks' pieces in rank order make the single-field stream, and rank 0's .asz equals what
asz_compress gives for the whole field. This serves fields larger than one GPU's memory.

The library calls back into the caller for its few exchanges (data range, default-slope samples,
the reconstructed planes below each slab before axis-0 rounds, the rerun decision, histograms and
the encoded pieces). `TorchComm` implements those callbacks with torch.distributed over host
tensors, so any backend with send/recv works (gloo on CPU hosts; on GPU hosts the halos are small
and go through host memory).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import api

ALLREDUCE = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_int)
ALLGATHER = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p)
SEND = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_uint64, C.c_int)
RECV = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_uint64, C.c_int)


class Comm(C.Structure):
    _fields_ = [("rank", C.c_int), ("size", C.c_int), ("user", C.c_void_p), ("allreduce", ALLREDUCE),
                ("allgather", ALLGATHER), ("send", SEND), ("recv", RECV)]


_DTYPES = {0: (C.c_float, np.float32), 1: (C.c_uint64, np.int64), 2: (C.c_int32, np.int32)}


def _view(ptr, n, ctype, np_dtype):
    return np.ctypeslib.as_array((ctype * n).from_address(ptr)).view(np_dtype)


class TorchComm:
    """asz_comm callbacks over torch.distributed (an initialised default process group). Buffers are
    wrapped as host tensors without copies; a failing collective returns 1 to the library."""

    def __init__(self, dist=None):
        if dist is None:
            import torch.distributed as dist
        self.dist = dist
        self.rank = dist.get_rank()
        self.size = dist.get_world_size()
        self._cb = (ALLREDUCE(self._allreduce), ALLGATHER(self._allgather), SEND(self._send), RECV(self._recv))
        self.struct = Comm(self.rank, self.size, None, *self._cb)

    def _tensor(self, ptr, nbytes):
        import torch
        return torch.from_numpy(_view(ptr, nbytes, C.c_uint8, np.uint8))

    def _allreduce(self, user, buf, count, dtype, op):
        try:
            import torch
            ctype, npt = _DTYPES[dtype]
            t = torch.from_numpy(_view(buf, count, ctype, npt))
            ops = {0: self.dist.ReduceOp.SUM, 1: self.dist.ReduceOp.MIN, 2: self.dist.ReduceOp.MAX}
            self.dist.all_reduce(t, op=ops[op])
            return 0
        except Exception:
            return 1

    def _allgather(self, user, send, nbytes, recv):
        try:
            src = self._tensor(send, nbytes).clone()
            outs = [self._tensor(recv + r * nbytes, nbytes) for r in range(self.size)] if nbytes else []
            if nbytes:
                tmp = [o.clone() for o in outs]
                self.dist.all_gather(tmp, src)
                for o, t in zip(outs, tmp):
                    o.copy_(t)
            else:
                self.dist.barrier()
            return 0
        except Exception:
            return 1

    def _send(self, user, buf, nbytes, dst):
        try:
            self.dist.send(self._tensor(buf, nbytes).clone(), dst)
            return 0
        except Exception:
            return 1

    def _recv(self, user, buf, nbytes, src):
        try:
            t = self._tensor(buf, nbytes)
            tmp = t.clone()
            self.dist.recv(tmp, src)
            t.copy_(tmp)
            return 0
        except Exception:
            return 1


def split_blocks(blocks0: int, world: int) -> list[tuple[int, int]]:
    """Contiguous axis-0 block ranges, one per rank, as even as the count allows (the first ranks take
    one more when it does not divide)."""
    if world < 1 or blocks0 < world:
        raise ValueError(f"{blocks0} axis-0 blocks cannot be shared by {world} ranks")
    q, r = divmod(blocks0, world)
    out, b = [], 0
    for k in range(world):
        n = q + (1 if k < r else 0)
        out.append((b, b + n))
        b += n
    return out


def slab_planes(dims, plan: str, block_begin: int, block_end: int, params: api.Params | None = None):
    """(plane_begin, plane_count, blocks0): the axis-0 planes a rank passes for its blocks."""
    L = api.lib()
    pb, pc, nb = C.c_uint64(), C.c_uint64(), C.c_uint64()
    rc = L.asz_slab_planes(api._dims(dims), C.byref(params) if params is not None else None, plan.encode(),
                           int(block_begin), int(block_end), C.byref(pb), C.byref(pc), C.byref(nb))
    if rc != api.ASZ_OK:
        raise api.AszError(rc, f"slab blocks [{block_begin}, {block_end}) do not fit the field")
    return pb.value, pc.value, nb.value


def blocks_of(dims, plan: str, params: api.Params | None = None) -> int:
    """The field's number of axis-0 blocks under the plan."""
    return slab_planes(dims, plan, 0, 1, params)[2]


def compress_slab(ctx: api.Context, comm: TorchComm, planes, dims, block_begin: int, block_end: int, rel_eb: float,
                  plan: str, family: str, params: api.Params | None = None):
    """Compress this rank's slab (NumPy planes, or a contiguous float32 CUDA tensor on the context's
    device). Returns (.asz bytes on rank 0 or None elsewhere, Report of the whole field)."""
    L = api.lib()
    p = params if params is not None else api.default_params()
    p.predictor_family = api._family_code(family)
    out = C.POINTER(C.c_uint8)()
    n = C.c_size_t(0)
    rep = api.Report()
    if api._is_cuda_tensor(planes):
        api._check_device_field(planes, ctx.device, "slab planes")
        ctx._use_torch_stream(planes)
        rc = L.asz_compress_slab(ctx._c, C.byref(comm.struct), C.c_void_p(planes.data_ptr()), 1, api._dims(dims),
                                 int(block_begin), int(block_end), C.c_float(rel_eb), C.byref(p), plan.encode(),
                                 C.byref(out), C.byref(n), C.byref(rep))
        L.asz_set_stream(ctx._c, None)
    else:
        a = np.ascontiguousarray(planes, dtype=np.float32)
        rc = L.asz_compress_slab(ctx._c, C.byref(comm.struct), C.c_void_p(a.ctypes.data), 0, api._dims(dims),
                                 int(block_begin), int(block_end), C.c_float(rel_eb), C.byref(p), plan.encode(),
                                 C.byref(out), C.byref(n), C.byref(rep))
    ctx._check(rc)
    if not out:
        return None, rep
    try:
        return C.string_at(out, n.value), rep
    finally:
        L.asz_free(out)
