"""The reference's own launcher drives this build's front ends as it drives the reference's.

t1_start_compressors.py:run_asz (:482-542) builds the command lines, runs s1_compress and
s1_decompress, parses their stdout (:256-290, :382-404), recomputes max error and PSNR from the
files, rejects an error above eb + 1 % and a reported CR that disagrees with the file size
(:517-523). This test imports that module from the reference sources (CPU only; skipped where they
are absent) with a stand-in for its `run_command` (its submodule is empty), and runs run_asz on the
cases of tests/golden/cli_cases.py twice:

* with the reference binaries (oracle/_ref, built from the reference's sources), run live;
* with this build's binaries, replayed from tests/golden/cli/asz_b200: the stdout, .asz and
  reconstruction that bin/s1_compress and bin/s1_decompress produced on a GPU host for the same
  command lines (recorded by cli_cases.py; the live stdout check is tests/test_cli_stdout.py).

Both must pass the launcher's checks and give the same result dictionaries, timing keys aside.
"""
import importlib.util
import os
import shutil
import subprocess
import sys
import tempfile
import types
from pathlib import Path

import pytest

from conftest import GOLDEN, REFERENCE_DIR, ROOT

sys.path.insert(0, GOLDEN)
import cli_cases  # noqa: E402

LAUNCHER = os.path.join(REFERENCE_DIR, "t1_start_compressors.py")
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
OURS = os.path.join(GOLDEN, "cli", "asz_b200")
TIME_KEYS = {"data_range_time", "compression_time", "decompression_time", "generate_config_time",
             "get_default_slope_time", "predictor_family_selection_time", "preprocessing_time"}

pytestmark = pytest.mark.skipif(not os.path.exists(LAUNCHER), reason="reference launcher not present")


def load_launcher(run_command):
    for name in ("third_party", "third_party.run_command"):
        mod = types.ModuleType(name)
        mod.__path__ = []
        sys.modules[name] = mod
    stub = types.ModuleType("third_party.run_command.run_command")
    stub.run_command = run_command
    sys.modules["third_party.run_command.run_command"] = stub
    spec = importlib.util.spec_from_file_location("t1_start_compressors_under_test", LAUNCHER)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class Runner:
    """run_command stand-in: runs the reference binaries, or replays this build's recorded runs."""

    def __init__(self, mode, case_name):
        self.mode, self.case = mode, case_name
        self.commands = []

    def __call__(self, cmd):
        cmd = [str(c) for c in cmd]
        self.commands.append(cmd)
        prog = os.path.basename(cmd[0])
        if self.mode == "reference":
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(r.stderr)
            return r.stdout
        z, rec = cmd[cmd.index("-z") + 1], cmd[cmd.index("-o") + 1]
        if prog == "s1_compress":
            shutil.copyfile(os.path.join(OURS, self.case + ".asz"), z)
            return open(os.path.join(OURS, self.case + ".compress.txt")).read()
        shutil.copyfile(os.path.join(OURS, self.case + ".out.f32"), rec)
        return open(os.path.join(OURS, self.case + ".decompress.txt")).read()


def run_case(mode, case):
    name, inp, shape, rel_eb, preds, method = case
    runner = Runner(mode, name)
    L = load_launcher(runner)
    L.asz_executable_directory = Path(REF_BIN if mode == "reference" else os.path.join(ROOT, "asz_b200", "bin"))
    with tempfile.TemporaryDirectory() as wd:
        data = Path(wd) / (os.path.basename(inp) + ".f32")
        shutil.copyfile(os.path.join(GOLDEN, inp + ".f32"), data)
        task = {"data_shape": [str(s) for s in shape], "data_path": data}
        result, predictors, family = L.run_asz(task, rel_eb, preds, dict(method))
        z = str(L.codec_output_path(task, ".asz"))
        rec = str(L.codec_output_path(task, ".bin"))
        expect = cli_cases.commands(L.asz_executable_directory, data, shape, rel_eb, preds, method, z, rec)
    return result, predictors, family, runner.commands, [list(map(str, c)) for c in expect]


@pytest.mark.parametrize("case", cli_cases.CASES, ids=[c[0] for c in cli_cases.CASES])
def test_launcher_layout_restated(case):
    if not os.path.exists(os.path.join(REF_BIN, "s1_compress")):
        pytest.skip("reference binaries not built")
    _, _, _, ran, expect = run_case("reference", case)
    assert ran == expect


@pytest.mark.parametrize("case", cli_cases.CASES, ids=[c[0] for c in cli_cases.CASES])
def test_launcher_accepts_this_build(case):
    if not os.path.exists(os.path.join(REF_BIN, "s1_compress")):
        pytest.skip("reference binaries not built")
    if not os.path.exists(os.path.join(OURS, case[0] + ".compress.txt")):
        pytest.skip("this build's runs not recorded yet (cli_cases.py on a GPU host)")
    ref, ref_preds, ref_fam, _, _ = run_case("reference", case)
    ours, preds, fam, ran, expect = run_case("asz_b200", case)
    assert ran == expect
    assert (preds, fam) == (ref_preds, ref_fam)
    strip = lambda d: {k: v for k, v in d.items() if k not in TIME_KEYS}  # noqa: E731
    assert strip(ours) == strip(ref)
