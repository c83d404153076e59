"""Regenerate the prediction-sweep golden fixtures from the reference's sweep tool built from its
own sources (c_codes/s2_many_prediction.cpp).

Run where the reference is mounted and `make -C oracle ref` has built
oracle/_ref/s2_many_prediction (its csv_tools include points at oracle/csv_shim.h, which writes
every value at full precision). Each case stores its input field (<name>.f32) and, in
s2_sweep.json, the arguments, the reference's min/max lines and every row it wrote: predictor,
key (rel_eb and coefficients) and the BR, H1, RMSE, MAE, PSNR and SAMPLES columns, as lists. The fields
are small seeded synthetic fields (the reference's datasets are external and not available).
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

REF = os.path.join(ROOT, "oracle", "_ref", "s2_many_prediction")

CASES = [
    # name, shape, (kind, alpha, seed), family-or-stencil, rel_ebs, six grid, targets
    ("s2_grf_all", (14, 16, 18), ("grf", 11 / 3, 21), "all", "1e-3", "legacy", "legacy"),
    ("s2_c1_1d6r_aug_common", (13, 20, 17), ("c1", None, 22), "1d6r", "1e-2,1e-5", "augmented", "common"),
    ("s2_rough_1d4r_shared1d", (12, 12, 25), ("grf", 1.2, 23), "1d4r", "1e-6,1e-1", "legacy", "shared1d"),
    ("s2_grf_2d4r_common", (16, 14, 12), ("grf", 2.5, 24), "2d4r", "1e-3", "legacy", "common"),
    ("s2_slab_1d6r_transition", (12, 13, 14), ("slab", 3.0, 25), "1d6r1", "1e-3", "transition", "legacy"),
]

COLUMNS = ("BR", "H1", "RMSE", "MAE", "PSNR", "SAMPLES")


def make_field(shape, recipe):
    kind, alpha, seed = recipe
    rng = np.random.default_rng(seed)
    if kind == "grf":
        return fields.grf_field(shape, alpha, rng).astype(np.float32)
    if kind == "c1":
        return fields.c1_field(seed=seed, shape=shape, blobs=3)
    if kind == "slab":
        f = fields.grf_field(shape, alpha, rng)
        f[: shape[0] // 3] = 0.0
        return f.astype(np.float32)
    raise ValueError(kind)


def parse_rows(path):
    rows = {}
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            key, col, val = line.split("|")
            if col not in COLUMNS:
                continue
            r = rows.setdefault(key, {"key": [float(k) for k in key.split(";")]})
            r[col] = int(val) if col == "SAMPLES" else float(val)
    return [[r["key"]] + [r[c] for c in COLUMNS] for r in rows.values()]


def main():
    out = {"generator": "oracle/_ref/s2_many_prediction (reference sources, reference flags)",
           "row": ["key (rel_eb, coefficients)"] + list(COLUMNS), "cases": []}
    for name, shape, recipe, family, ebs, grid, targets in CASES:
        data = make_field(shape, recipe)
        data.tofile(os.path.join(HERE, name + ".f32"))
        with tempfile.TemporaryDirectory() as wd:
            prefix = os.path.join(wd, "out")
            r = subprocess.run([REF, os.path.join(HERE, name + ".f32"), *map(str, shape), prefix, family, ebs, grid, targets],
                               capture_output=True, text=True, check=True)
            preds = {}
            for fn in sorted(os.listdir(wd)):
                if fn.startswith("out_") and fn.endswith(".csv"):
                    preds[fn[4:-4]] = parse_rows(os.path.join(wd, fn))
        lines = r.stdout.splitlines()
        out["cases"].append({
            "name": name, "shape": list(shape), "family": family, "rel_ebs": ebs, "six_grid": grid, "targets": targets,
            "stdout_head": lines[:3], "rows": preds,
        })
        print(name, {k: len(v) for k, v in preds.items()})
    with open(os.path.join(HERE, "s2_sweep.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))


if __name__ == "__main__":
    main()
