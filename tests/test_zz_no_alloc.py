"""asz_error_stats_noalloc: the allocation-free error statistics.

Collected last (file name) so that it also runs after every other test has used the library's
contexts on the same device. Compared with asz_compress_stats on two calls in a row.
"""
import ctypes as C

import numpy as np
import pytest

import asz_b200.api as api
from asz_b200 import fields

# 65520 tiles of 65536 values: the fixed scratch limit stated in include/asz_b200.h.
MAX_VALUES = 65520 * 65536


def test_noalloc_rejects_oversize_before_touching_the_device():
    # Size checks come before any CUDA call, so this runs without a GPU; the pointers are never read.
    L = api.lib()
    err = C.create_string_buffer(256)
    m, ps = C.c_double(), C.c_double()
    rc = L.asz_error_stats_noalloc(C.c_void_p(16), C.c_void_p(16), MAX_VALUES + 1, 1.0, None, C.byref(m), C.byref(ps),
                                   err, 256)
    assert rc == api.ASZ_E_ARG
    assert b"exceed the fixed scratch limit" in err.value
    rc = L.asz_error_stats_noalloc(None, None, 10, 1.0, None, C.byref(m), C.byref(ps), err, 256)
    assert rc == api.ASZ_E_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(40, 48, 64), (130, 97, 65)])
def test_noalloc_matches_compress_stats(shape):
    import torch
    x_np = fields.c2_field(seed=11, shape=shape)
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(x_np).to(dev)
    ctx = api.Context(0)
    try:
        blob, rep = ctx.compress(x, 1e-3, ",".join(["cubic2_012"] * 5), "cubic", api.default_params(block_pivot_ratio=3))
        y = torch.empty_like(x)
        ctx.decompress(blob, shape, 1e-3, api.default_params(block_pivot_ratio=3), out=y)
        torch.cuda.synchronize(dev)
        value_range = float(rep.max_val) - float(rep.min_val)
        ref = [ctx.stats() for _ in range(2)]
        got = [api.error_stats_noalloc(x, y, value_range) for _ in range(2)]
    finally:
        ctx.close()
    # Fixed summation order: the two calls agree bit for bit.
    assert got[0] == got[1]
    for (m_ref, p_ref), (m, p) in zip(ref, got):
        assert m == m_ref
        # asz_compress_stats sums with atomics (any order); 1e-12 relative covers the reordering.
        assert abs(p - p_ref) <= 1e-12 * abs(p_ref)
    # The reference's bound is met up to float rounding of the reconstruction (it reports up to
    # about 100.001 % of eb itself).
    assert got[0][0] <= 1.001 * rep.abs_eb
    # An independent check of the figures in float64 on the host.
    yh = y.cpu().numpy()
    d = x_np.astype(np.float64) - yh.astype(np.float64)
    assert got[0][0] == float(np.abs(x_np - yh).max())
    psnr = 10 * np.log10(value_range ** 2 / np.mean(d * d))
    assert abs(got[0][1] - psnr) <= 1e-9 * abs(psnr)
