"""The CLI front ends print the reference's stdout, line for line.

The reference's launcher reads the compressor's and decompressor's stdout (t1_start_compressors.py
:256-290, :382-404), so the drop-in claim covers every printed line, not only the .asz. These tests
run bin/s1_compress and bin/s1_decompress with the launcher's command lines (tests/golden/
cli_cases.py) and compare their stdout with what the reference binaries printed for the same
command (tests/golden/cli/reference, and the full-size record in tests/golden/fullsize.json). Only
the wall-clock figures ("... time: <x> s" and the plan-search breakdown) are masked: every other
number, including max_err, CR, BR, PSNR and dist, must print the same digits.
"""
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

sys.path.insert(0, GOLDEN)
import cli_cases  # noqa: E402

BIN = os.path.join(ROOT, "asz_b200", "bin")
REF_DIR = os.path.join(GOLDEN, "cli", "reference")
TIME = re.compile(r"(?<![0-9A-Za-z_])[0-9]+\.[0-9]+ s\b")


def masked(text):
    return [TIME.sub("<t> s", ln) for ln in text.splitlines()]


def assert_same_lines(ours, ref, what):
    a, b = masked(ours), masked(ref)
    diff = [(i, x, y) for i, (x, y) in enumerate(zip(a, b)) if x != y]
    assert not diff and len(a) == len(b), f"{what}: first differences {diff[:4]} (lines {len(a)} vs {len(b)})"


def test_mask_keeps_non_time_numbers():
    assert masked("Compression time: 0.123456 s\nCR: 4.5, BR: 7.0\ndist=19.68") == [
        "Compression time: <t> s", "CR: 4.5, BR: 7.0", "dist=19.68"]
    assert masked("Generate config breakdown: statistics=0.010161 s,sample prediction=0.000185 s")[0] == \
        "Generate config breakdown: statistics=<t> s,sample prediction=<t> s"


@pytest.mark.gpu
@pytest.mark.parametrize("case", cli_cases.CASES, ids=[c[0] for c in cli_cases.CASES])
def test_cli_stdout_matches_reference(case):
    name, inp, shape, rel_eb, preds, method = case
    with tempfile.TemporaryDirectory() as wd:
        data = os.path.join(wd, os.path.basename(inp) + ".f32")
        shutil.copyfile(os.path.join(GOLDEN, inp + ".f32"), data)
        z, rec = os.path.join(wd, "o.asz"), os.path.join(wd, "o.out.f32")
        comp, dec = cli_cases.commands(BIN, data, shape, rel_eb, preds, method, z, rec)
        rc = subprocess.run(comp, capture_output=True, text=True)
        assert rc.returncode == 0, rc.stderr
        rd = subprocess.run(dec, capture_output=True, text=True)
        assert rd.returncode == 0, rd.stderr
        with open(z, "rb") as f:
            blob = f.read()
        with open(os.path.join(REF_DIR, name + ".asz"), "rb") as f:
            assert blob == f.read(), ".asz differs from the reference's"
        assert_same_lines(rc.stdout, open(os.path.join(REF_DIR, name + ".compress.txt")).read(), "s1_compress")
        assert_same_lines(rd.stdout, open(os.path.join(REF_DIR, name + ".decompress.txt")).read(), "s1_decompress")
        x = np.fromfile(data, np.float32)
        y = np.fromfile(rec, np.float32)
        assert x.shape == y.shape


FULL = json.load(open(os.path.join(GOLDEN, "fullsize.json")))
FULL_CASES = ["c1_auto_1e-03_bpr3", "c2_quintic_1e-05"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", FULL_CASES)
def test_cli_stdout_matches_reference_at_full_size(name):
    import make_fullsize
    case = next(c for c in FULL["cases"] if c["name"] == name)
    x = make_fullsize.make_field(case["field"])
    if make_fullsize.sha(x.tobytes()) != FULL["fields"][case["field"]]["sha256"]:
        pytest.skip("generated input differs from the recorded one (other NumPy build)")
    with tempfile.TemporaryDirectory() as wd:
        inp = os.path.join(wd, "in.f32")
        x.tofile(inp)
        del x
        z, rec = os.path.join(wd, "o.asz"), os.path.join(wd, "o.out")
        argv = case["compress_argv"]
        # The recorded command with this run's paths and binary.
        args = argv[1:]
        args[args.index("-i") + 1] = inp
        args[args.index("-z") + 1] = z
        args[args.index("-o") + 1] = rec
        rc = subprocess.run([os.path.join(BIN, "s1_compress"), *args], capture_output=True, text=True)
        assert rc.returncode == 0, rc.stderr
        dargs = [a for a in args]
        if "--predictor-plan" in dargs:
            k = dargs.index("--predictor-plan")
            del dargs[k:k + 2]
        rd = subprocess.run([os.path.join(BIN, "s1_decompress"), *dargs], capture_output=True, text=True)
        assert rd.returncode == 0, rd.stderr
        assert_same_lines(rc.stdout, case["stdout_compress"], "s1_compress")
        assert_same_lines(rd.stdout, case["stdout_decompress"], "s1_decompress")
