"""The C ABI: the library loads and exports every entry point include/asz_b200.h declares; the
CLI front ends reject bad arguments the way the reference does. No GPU needed."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

LIB = os.path.join(ROOT, "asz_b200", "libasz_b200.so")
HDR = os.path.join(ROOT, "include", "asz_b200.h")
BIN = os.path.join(ROOT, "asz_b200", "bin")


def declared_functions():
    text = open(HDR).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(asz_[a-z_0-9]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ["asz_create", "asz_destroy", "asz_compress", "asz_decompress", "asz_last_error", "asz_free",
              "asz_default_params", "asz_set_stream"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_default_params_match_reference_defaults():
    import asz_b200.api as api
    p = api.default_params()
    assert (p.pivot_eb_ratio, p.eb_ratio, p.slope_ratio) == pytest.approx((0.05, 0.76, 0.54))
    assert p.block_pivot_ratio == 4 and p.max_layer_num == 14 and p.t_precision == 32
    assert p.h1_block_sampling_num == 256 and p.stat_eb_ratio == pytest.approx(0.2)
    assert p.predictor_family == api.ASZ_FAMILY_AUTO


@pytest.mark.parametrize("args,msg", [
    (["--bogus"], "error: unknown argument: --bogus"),
    (["-i", "x.f32", "-3", "7", "7", "6", "-M", "REL", "1e-3"], "error: all three dimensions must be at least 7"),
    (["-i", "x.f32", "-3", "8", "8", "8", "-M", "REL", "0"], "error: relative error bound must be positive and finite"),
    (["--predictor-family", "sextic"], "error: predictor_family must be cubic or quintic"),
])
def test_cli_argument_errors(args, msg):
    r = subprocess.run([os.path.join(BIN, "s1_compress"), *args], capture_output=True, text=True)
    assert r.returncode == 1
    assert r.stderr.strip() == msg


@pytest.mark.gpu
def test_output_blocks_are_reused_and_released(gpu_ctx):
    """Output buffers released with asz_free serve later outputs (single and batched calls give
    the same bytes again), and asz_release_output_cache empties the cache between calls."""
    import numpy as np

    import asz_b200.api as api
    from asz_b200 import fields
    rng = np.random.default_rng(9)
    a = fields.grf_field((40, 36, 44), 3.0, rng).astype(np.float32)
    b = fields.grf_field((24, 30, 20), 2.0, rng).astype(np.float32)
    p = api.default_params(block_pivot_ratio=3)
    plan = "cubic0_012,cubic1_012,cubic2_012"
    first = [gpu_ctx.compress(x, 1e-3, plan, "cubic", p)[0] for x in (a, b, a)]
    assert first[0] == first[2]
    again = [gpu_ctx.compress(x, 1e-3, plan, "cubic", p)[0] for x in (b, a)]
    assert again == [first[1], first[0]]
    blobs, _, _ = gpu_ctx.compress_batch([a, b], 1e-3, plan, "cubic", p)
    assert blobs == [first[0], first[1]]
    api.lib().asz_release_output_cache()
    assert gpu_ctx.compress(a, 1e-3, plan, "cubic", p)[0] == first[0]


def _bare_context(device=0):
    # A Context object that never reached asz_create: any library call through it would fail,
    # so these tests show that the argument checks run first.
    import asz_b200.api as api
    ctx = object.__new__(api.Context)
    ctx._L = None
    ctx._c = None
    ctx.device = device
    return ctx


def test_decompress_refuses_a_host_out_tensor():
    import torch
    ctx = _bare_context()
    with pytest.raises(ValueError, match="CUDA tensor"):
        ctx.decompress(b"\0" * 16, (8, 8, 8), 1e-3, params=None, out=torch.empty(512))


@pytest.mark.parametrize("case", ["dtype", "strided", "device", "numel"])
def test_device_buffer_checks(case):
    import torch
    import asz_b200.api as api
    x = torch.empty(8, 8, 8, dtype=torch.float32)
    numel = 512
    if case == "dtype":
        x = x.double()
    elif case == "strided":
        x = x.transpose(0, 2)
    elif case == "numel":
        numel = 1000
    # A host tensor reports no device index, so it fails the device check of any context.
    with pytest.raises(ValueError):
        api._check_device_field(x, 0, "out", numel)
