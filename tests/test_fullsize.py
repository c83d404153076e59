"""Parity at the benchmark sizes: the GPU path against the reference compressor's own output.

tests/golden/fullsize.json holds, for each configuration, SHA-256 digests of what the reference
binaries (built from the reference's sources, tests/golden/make_fullsize.py) produced for the same
seeded input: the .asz, the stream before zstd and the decompressed float32. The cases are the
512^3 C2 field at REL 1e-2, 1e-3, 1e-4 and 1e-5 with the plan cubic2_012 on all 9 levels in both
predictor families (block pivot ratio 3, or 96 at REL <= 1e-4, the launcher's rule), and the
100x500x500 C1 field with the compressor's own plan search and family selection (block pivot ratio
3 and the binary's default 4). Reference behaviour held: compress.tpp:147-321, decompress.tpp:79-208.

The inputs are generated on the host from their seeds. If the generated bytes differ from the
recorded input digest (another NumPy build), the reference binaries in oracle/_ref are run on the
generated bytes instead, when present.
"""
import hashlib
import json
import os
import sys
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

sys.path.insert(0, GOLDEN)

FIX_PATH = os.path.join(GOLDEN, "fullsize.json")
FIX = json.load(open(FIX_PATH)) if os.path.exists(FIX_PATH) else {"fields": {}, "cases": []}
CASES = {c["name"]: c for c in FIX["cases"]}


def sha(b) -> str:
    return hashlib.sha256(b).hexdigest()


@pytest.fixture(scope="module")
def field_cache():
    cache = {}

    def get(key):
        if key not in cache:
            cache.clear()  # one 512 MiB field at a time
            import make_fullsize
            x = make_fullsize.make_field(key)
            cache[key] = (x, sha(x.tobytes()))
        return cache[key]

    return get


def expected_for(case, x, digest):
    """The recorded digests, or the reference binaries' live digests when the input differs."""
    if digest == FIX["fields"][case["field"]]["sha256"]:
        return case
    import make_fullsize
    import oracle as O
    if O.ref_binary("s1_compress") is None:
        pytest.fail(f"generated {case['field']} input differs from the recorded one and oracle/_ref is absent")
    spec = (case["name"], case["field"], case["rel_eb"], case["plan"], case["family"], case["block_pivot_ratio"])
    with tempfile.TemporaryDirectory() as wd:
        inp = os.path.join(wd, "in.f32")
        x.tofile(inp)
        return make_fullsize.run_case(spec, inp, x.shape, wd)


def report(name, rec):
    out_dir = os.environ.get("ASZ_TEST_REPORT_DIR")
    if out_dir:
        os.makedirs(out_dir, exist_ok=True)
        with open(os.path.join(out_dir, f"fullsize_{name}.json"), "w") as f:
            json.dump(rec, f)
    print(json.dumps(rec))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_fullsize_matches_reference(name, gpu_ctx, field_cache):
    import asz_b200.api as api
    case = CASES[name]
    x, digest = field_cache(case["field"])
    exp = expected_for(case, x, digest)
    p = api.default_params()
    if case["block_pivot_ratio"] is not None:
        p.block_pivot_ratio = case["block_pivot_ratio"]
    blob, rep = gpu_ctx.compress(x, case["rel_eb"], case["plan"], case["family"] or "auto", p)
    pre = gpu_ctx.debug_pre_zstd()
    dec, _ = gpu_ctx.decompress(blob, x.shape, case["rel_eb"], p)
    max_err = float(np.abs(x.astype(np.float64) - dec.astype(np.float64)).max())
    rec = {"case": name, "asz_len": len(blob), "cr": x.nbytes / len(blob), "plan": rep.plan.decode(),
           "family": "quintic" if rep.quintic else "cubic", "exact_groups": int(rep.exact_groups),
           "serial_groups": int(rep.serial_groups), "ambiguous_decisions": int(rep.ambiguous_decisions),
           "reruns": int(rep.reruns), "t_fallback_count": int(rep.t_fallback_count),
           "max_err_over_abs_eb": max_err / float(rep.abs_eb),
           "input_digest_recorded": exp is case}
    report(name, rec)
    assert len(blob) == exp["asz_len"]
    assert sha(pre) == exp["pre_zstd_sha256"], "stream before zstd differs from the reference's"
    assert sha(blob) == exp["asz_sha256"], ".asz differs from the reference's (same libzstd)"
    assert sha(dec.tobytes()) == exp["decompressed_sha256"], "decompressed float32 differs from s1_decompress"
    # The launcher's acceptance (t1_start_compressors.py:458-459): max error within eb plus 1 %.
    assert max_err <= 1.01 * float(rep.abs_eb)
    assert abs(rec["max_err_over_abs_eb"] - exp["max_err_over_abs_eb"]) <= 1e-6
