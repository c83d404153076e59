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
