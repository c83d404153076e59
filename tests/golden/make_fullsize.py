"""Full-size golden record: the reference compressor on the benchmark configurations.

Run where the reference is mounted and `make -C oracle ref` has built oracle/_ref (the reference
compiled from its own sources with its own flags). For each case it generates the seeded field
(asz_b200.fields, NumPy on the host), runs the reference's s1_compress and s1_decompress with the
launcher's argument layout (t1_start_compressors.py:486-510: -f -i -3 -M REL %.17g, block pivot
ratio 3 above REL 1e-4 and 96 at or below it) and records SHA-256 digests of the input, the .asz,
the stream before zstd and the decompressed output, with the reference's stdout lines. The fields
are 100 MB to 512 MiB, too large to commit; their digests are small and pin the reference's
output for the same bytes, so tests/test_fullsize.py can hold the GPU path to it.

    python tests/golden/make_fullsize.py          # writes tests/golden/fullsize.json (minutes)
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes as C
import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
from asz_b200 import fields  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.join(HERE, "fullsize.json")

C2_PLAN = ",".join(["cubic2_012"] * 9)

# name, field, rel_eb, plan (None: the compressor's plan search), family (None: its selector),
# block_pivot_ratio (None: the binary's default of 4).
CASES = []
for _rel in (1e-2, 1e-3, 1e-4, 1e-5):
    for _fam in ("cubic", "quintic"):
        CASES.append((f"c2_{_fam}_{_rel:g}", "c2", _rel, C2_PLAN, _fam, 3 if _rel > 1e-4 else 96))
CASES.append(("c1_auto_1e-03_bpr3", "c1", 1e-3, None, None, 3))
CASES.append(("c1_auto_1e-03_bpr4", "c1", 1e-3, None, None, None))

FIELDS = {
    "c2": {"recipe": "asz_b200.fields.c2_field(seed=2)", "shape": [512, 512, 512]},
    "c1": {"recipe": "asz_b200.fields.c1_field(seed=1)", "shape": [100, 500, 500]},
}


def make_field(key):
    if key == "c2":
        return fields.c2_field(seed=2)
    if key == "c1":
        return fields.c1_field(seed=1)
    raise ValueError(key)


def sha(b) -> str:
    return hashlib.sha256(b).hexdigest()


def zstd_decompress(blob: bytes) -> bytes:
    z = C.CDLL("libzstd.so.1")
    z.ZSTD_getFrameContentSize.restype = C.c_ulonglong
    z.ZSTD_getFrameContentSize.argtypes = [C.c_void_p, C.c_size_t]
    z.ZSTD_decompress.restype = C.c_size_t
    z.ZSTD_decompress.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t]
    n = z.ZSTD_getFrameContentSize(blob, len(blob))
    out = C.create_string_buffer(n)
    got = z.ZSTD_decompress(out, n, blob, len(blob))
    assert got == n
    return out.raw[:n]


def common_args(shape, rel_eb, case):
    _, _, _, plan, family, bpr = case
    args = ["-f", "-3", *map(str, shape), "-M", "REL", f"{rel_eb:.17g}"]
    if bpr is not None:
        args += ["--block-pivot-ratio", str(bpr)]
    if family is not None:
        args += ["--predictor-family", family]
    return args


def run_case(case, inp, shape, wd):
    name, _, rel_eb, plan, family, bpr = case
    z = os.path.join(wd, name + ".asz")
    rec = os.path.join(wd, name + ".out")
    common = common_args(shape, rel_eb, case)
    comp = [os.path.join(REF, "s1_compress"), "-i", inp, *common, "-z", z, "-o", rec]
    if plan:
        comp += ["--predictor-plan", plan]
    t0 = time.perf_counter()
    rc = subprocess.run(comp, capture_output=True, text=True, check=True)
    comp_s = time.perf_counter() - t0
    dec = [os.path.join(REF, "s1_decompress"), "-i", inp, *common, "-z", z, "-o", rec]
    t0 = time.perf_counter()
    rd = subprocess.run(dec, capture_output=True, text=True, check=True)
    dec_s = time.perf_counter() - t0
    with open(z, "rb") as f:
        blob = f.read()
    pre = zstd_decompress(blob)
    out = np.fromfile(rec, np.float32)
    data = np.fromfile(inp, np.float32)
    max_err = float(np.abs(data.astype(np.float64) - out.astype(np.float64)).max())
    rng = float(data.max()) - float(data.min())
    os.unlink(rec)
    os.unlink(z)
    return {
        "name": name, "field": case[1], "rel_eb": rel_eb, "plan": plan, "family": family, "block_pivot_ratio": bpr,
        "compress_argv": [os.path.basename(comp[0])] + comp[1:],
        "asz_sha256": sha(blob), "asz_len": len(blob), "pre_zstd_sha256": sha(pre), "pre_zstd_len": len(pre),
        "decompressed_sha256": sha(out.tobytes()), "max_err_over_abs_eb": max_err / (rel_eb * rng),
        "reference_wall_s": {"compress": comp_s, "decompress": dec_s},
        "stdout_compress": rc.stdout, "stdout_decompress": rd.stdout,
    }


def main():
    jobs = int(os.environ.get("JOBS", str(os.cpu_count() or 4)))
    record = {"generator": "tests/golden/make_fullsize.py", "reference": "oracle/_ref (s1_compress, s1_decompress)",
              "gxx": subprocess.run(["g++", "--version"], capture_output=True, text=True).stdout.splitlines()[0],
              "fields": {}, "cases": []}
    with tempfile.TemporaryDirectory() as wd:
        inputs = {}
        for key, meta in FIELDS.items():
            f = make_field(key)
            path = os.path.join(wd, key + ".f32")
            f.tofile(path)
            inputs[key] = (path, f.shape)
            record["fields"][key] = {**meta, "sha256": sha(f.tobytes())}
            del f
        with cf.ThreadPoolExecutor(jobs) as ex:
            futs = [ex.submit(run_case, c, inputs[c[1]][0], inputs[c[1]][1], wd) for c in CASES]
            for fu in futs:
                r = fu.result()
                record["cases"].append(r)
                print(r["name"], r["asz_len"], f"{r['reference_wall_s']['compress']:.1f}s", flush=True)
    with open(OUT, "w") as f:
        json.dump(record, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
