"""Command lines of the reference's launcher for a few small cases, and a recorder for their outputs.

The launcher (t1_start_compressors.py:482-542, run_asz) runs s1_compress and then s1_decompress
with one argument layout: "-f -i DATA -3 D0 D1 D2 -M REL <rel_eb %.17g>", the method's options
in its fixed key order (block pivot ratio 96 at REL <= 1e-4, else 3, unless the method sets it),
"--predictor-family" when given, then "-z COMPRESSED -o RECONSTRUCTED", the compress-only options,
"--report-t-histogram" and "--predictor-plan". `commands` restates that layout so the recorded
outputs are those the launcher would see; tests/test_launcher.py checks the restatement against
the launcher's own command lines.

    python tests/golden/cli_cases.py --binaries oracle/_ref --out tests/golden/cli/reference --no-recon
    python tests/golden/cli_cases.py --binaries asz_b200/bin --out <dir>      # on a GPU host

Each case leaves <name>.compress.txt and <name>.decompress.txt (stdout), <name>.asz and
(without --no-recon) <name>.out.f32 in the output directory.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))

# name, input (tests/golden/<input>.f32; cli/c1_24x40x40 is fields.c1_field(seed=21, blobs=4) at
# that shape, the smallest C1-like field on which the family selector samples blocks), shape,
# rel_eb, predictors (None: plan search), the launcher's method options.
CASES = [
    ("grf53_plan_cubic", "grf53_cubic2x3", (20, 24, 30), 1e-3, ["cubic2_012"] * 3, {"predictor_family": "cubic"}),
    ("c1_auto_1e-3", "cli/c1_24x40x40", (24, 40, 40), 1e-3, None, {}),
    ("c1_auto_1e-5", "cli/c1_24x40x40", (24, 40, 40), 1e-5, None, {}),
    ("c2like_quintic_hist", "c2like_quintic", (32, 32, 32), 1e-4, ["cubic2_012"] * 5,
     {"predictor_family": "quintic", "report_t_histogram": True}),
    ("c1_options_1e-2", "cli/c1_24x40x40", (24, 40, 40), 1e-2, None,
     {"predictor_family": "cubic", "block_pivot_ratio": 4, "stat_eb_ratio": 0.3, "h1_block_sampling_num": 128,
      "eb_ratio": 0.9}),
]

OPTION_NAMES = {
    "pivot_eb_ratio": "--pivot-eb-ratio", "eb_ratio": "--eb-ratio", "slope_ratio": "--slope-ratio",
    "block_pivot_ratio": "--block-pivot-ratio", "max_layer_num": "--max-layer-num",
    "full_predictor_search_layer_num": "--full-predictor-search-layer-num",
    "generate_config_sample_stride": "--generate-config-sample-stride",
    "h1_block_sampling_num": "--h1-block-sampling-num", "stat_eb_ratio": "--stat-eb-ratio",
    "predictor_family_suffix_layers": "--predictor-family-suffix-layers",
    "predictor_family_sample_blocks": "--predictor-family-sample-blocks",
    "predictor_family_sample_point_limit": "--predictor-family-sample-point-limit",
    "predictor_family_sample_fraction_limit": "--predictor-family-sample-fraction-limit",
    "predictor_family_coarse_probe_block_pivot_ratio": "--predictor-family-coarse-probe-block-pivot-ratio",
    "predictor_family_fine_probe_block_pivot_ratio": "--predictor-family-fine-probe-block-pivot-ratio",
    "predictor_family_fine_eb_threshold": "--predictor-family-fine-eb-threshold",
    "default_slope_invalid_ratio_threshold": "--default-slope-invalid-ratio-threshold",
    "default_slope_fallback": "--default-slope-fallback", "default_slope_eb_span": "--default-slope-eb-span",
    "t_precision": "--t-precision", "t_min": "--t-min", "t_max": "--t-max",
}
COMMON_KEYS = ("pivot_eb_ratio", "eb_ratio", "slope_ratio", "block_pivot_ratio", "max_layer_num",
               "full_predictor_search_layer_num", "t_precision")
COMPRESS_KEYS = ("generate_config_sample_stride", "h1_block_sampling_num", "stat_eb_ratio",
                 "predictor_family_suffix_layers", "predictor_family_sample_blocks",
                 "predictor_family_sample_point_limit", "predictor_family_sample_fraction_limit",
                 "predictor_family_coarse_probe_block_pivot_ratio", "predictor_family_fine_probe_block_pivot_ratio",
                 "predictor_family_fine_eb_threshold", "default_slope_invalid_ratio_threshold",
                 "default_slope_fallback", "default_slope_eb_span", "t_min", "t_max")


def commands(bindir, data, shape, rel_eb, predictors, method, z, rec):
    """(compress argv, decompress argv) in the launcher's layout."""
    opts = dict(method)
    opts.setdefault("block_pivot_ratio", 96 if rel_eb <= 1e-4 else 3)
    common = ["-f", "-i", str(data), "-3", *[str(s) for s in shape], "-M", "REL", f"{rel_eb:.17g}"]
    for k in COMMON_KEYS:
        if k in opts:
            common += [OPTION_NAMES[k], str(opts[k])]
    if "predictor_family" in opts:
        common += ["--predictor-family", str(opts["predictor_family"])]
    comp = [os.path.join(str(bindir), "s1_compress"), *common, "-z", str(z), "-o", str(rec)]
    for k in COMPRESS_KEYS:
        if k in opts:
            comp += [OPTION_NAMES[k], str(opts[k])]
    if opts.get("report_t_histogram", False):
        comp.append("--report-t-histogram")
    if predictors is not None:
        comp += ["--predictor-plan", ",".join(predictors)]
    dec = [os.path.join(str(bindir), "s1_decompress"), *common, "-z", str(z), "-o", str(rec)]
    return comp, dec


def record(bindir, out_dir, names=None, keep_recon=True):
    os.makedirs(out_dir, exist_ok=True)
    with tempfile.TemporaryDirectory() as wd:
        for name, inp, shape, rel_eb, preds, method in CASES:
            if names and name not in names:
                continue
            data = os.path.join(wd, os.path.basename(inp) + ".f32")
            shutil.copyfile(os.path.join(HERE, inp + ".f32"), data)
            z, rec = os.path.join(wd, name + ".asz"), os.path.join(wd, name + ".out.f32")
            comp, dec = commands(bindir, data, shape, rel_eb, preds, method, z, rec)
            rc = subprocess.run(comp, capture_output=True, text=True, check=True)
            rd = subprocess.run(dec, capture_output=True, text=True, check=True)
            with open(os.path.join(out_dir, name + ".compress.txt"), "w") as f:
                f.write(rc.stdout)
            with open(os.path.join(out_dir, name + ".decompress.txt"), "w") as f:
                f.write(rd.stdout)
            shutil.copyfile(z, os.path.join(out_dir, name + ".asz"))
            if keep_recon:
                shutil.copyfile(rec, os.path.join(out_dir, name + ".out.f32"))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--binaries", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--no-recon", action="store_true", help="keep stdout and .asz only")
    a = ap.parse_args()
    record(os.path.abspath(a.binaries), os.path.abspath(a.out), keep_recon=not a.no_recon)
