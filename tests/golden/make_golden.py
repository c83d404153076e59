"""Regenerate the golden fixtures from the reference compressor built from its own sources.

Run in a container where the reference is mounted and `make -C oracle ref` has built
oracle/_ref/{s1_compress,s1_decompress}. Each case stores the input field, the reference's .asz,
its decompressed output and the arguments, listed in manifest.json. The fields are small seeded
synthetic fields (the reference's datasets are external and not available).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
from asz_b200 import fields  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")

CASES = [
    # name, shape, field recipe, rel_eb, plan, family, block_pivot_ratio
    ("grf53_cubic2x3", (20, 24, 30), ("grf", 5 / 3, 11), 1e-3, "cubic2_012,cubic2_012,cubic2_012", "cubic", 3),
    ("grf113_mixed", (33, 17, 40), ("grf", 11 / 3, 12), 1e-2,
     "cubic0_120,cubic1_021,cubic2_012,cubic0_012,cubic1_012,cubic2_120", "quintic", 4),
    ("c1like_cyclic", (25, 30, 30), ("c1", None, 13), 1e-3,
     "cubic0_012,cubic1_012,cubic2_012,cubic0_012,cubic1_012,cubic2_012", "cubic", 3),
    ("c2like_quintic", (32, 32, 32), ("c2", None, 14), 1e-4, ",".join(["cubic2_012"] * 5), "quintic", 96),
    ("flat_slab_min7", (7, 9, 16), ("slab", 3.0, 15), 1e-3, "cubic2_021,cubic1_120", "cubic", 1),
    ("rough_1e5", (18, 18, 18), ("grf", 1.2, 16), 1e-5, "cubic1_021,cubic0_120,cubic2_012", "cubic", 2),
]


def make_field(shape, recipe):
    kind, alpha, seed = recipe
    rng = np.random.default_rng(seed)
    if kind == "grf":
        return fields.grf_field(shape, alpha, rng).astype(np.float32)
    if kind == "c1":
        return fields.c1_field(seed=seed, shape=shape, blobs=4)
    if kind == "c2":
        return fields.c2_field(seed=seed, shape=shape)
    if kind == "slab":
        f = fields.grf_field(shape, alpha, rng)
        f[: shape[0] // 2] = 0.0
        return f.astype(np.float32)
    raise ValueError(kind)


def main():
    manifest = []
    for name, shape, recipe, eb, plan, family, bpr in CASES:
        data = make_field(shape, recipe)
        with tempfile.TemporaryDirectory() as wd:
            inp = os.path.join(wd, "in.f32")
            z = os.path.join(wd, "out.asz")
            o = os.path.join(wd, "out.f32")
            data.tofile(inp)
            dims = [str(s) for s in shape]
            extra = ["--predictor-plan", plan, "--predictor-family", family, "--block-pivot-ratio", str(bpr)]
            subprocess.run([os.path.join(REF, "s1_compress"), "-i", inp, "-z", z, "-3", *dims, "-M", "REL", repr(eb),
                            *extra], check=True, capture_output=True)
            subprocess.run([os.path.join(REF, "s1_decompress"), "-z", z, "-o", o, "-3", *dims, "-M", "REL", repr(eb),
                            "--block-pivot-ratio", str(bpr)], check=True, capture_output=True)
            data.tofile(os.path.join(HERE, f"{name}.f32"))
            with open(z, "rb") as f:
                blob = f.read()
            with open(os.path.join(HERE, f"{name}.asz"), "wb") as f:
                f.write(blob)
            rec = np.fromfile(o, np.float32)
            rec.tofile(os.path.join(HERE, f"{name}.out.f32"))
        manifest.append(dict(name=name, shape=list(shape), rel_eb=eb, plan=plan, family=family,
                             block_pivot_ratio=bpr))
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(dict(generator="oracle/_ref s1_compress/s1_decompress (reference built from source)",
                       cases=manifest), f, indent=1)


if __name__ == "__main__":
    main()
