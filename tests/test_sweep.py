"""The prediction sweep (s2_many_prediction): the CPU oracle against the reference tool's golden
rows and against the reference's own functions; the kernel's target mapping and the coefficient
grids against the oracle (host-side, no GPU); the CUDA sweep against the golden rows and the
oracle (QB-derived figures exact, sums to 1e-12 relative); the command-line front end."""
import json
import os
import subprocess
import sys
import ctypes as C

import numpy as np
import pytest

import oracle as O

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
GOLDEN = os.path.join(ROOT, "tests", "golden")
CLI = os.path.join(ROOT, "asz_b200", "bin", "s2_many_prediction")
EXACT = ("BR", "H1", "SAMPLES")
SUMS = ("RMSE", "MAE", "PSNR")
SUM_RTOL = 1e-12


def _golden():
    with open(os.path.join(GOLDEN, "s2_sweep.json")) as f:
        g = json.load(f)
    for case in g["cases"]:
        data = np.fromfile(os.path.join(GOLDEN, case["name"] + ".f32"), np.float32).reshape(case["shape"])
        yield case, data, g["row"][1:]


def _cols(r):
    return {"BR": r.br, "H1": r.h1, "RMSE": r.rmse, "MAE": r.mae, "PSNR": r.psnr, "SAMPLES": r.samples}


def _rng_field(rng, shape, rough=False):
    from asz_b200 import fields
    f = fields.grf_field(shape, rng.uniform(1.2, 2.0) if rough else rng.uniform(2.5, 4.5), rng)
    return (f * rng.uniform(0.5, 50) + rng.uniform(-10, 10)).astype(np.float32)


# ---------------------------------------------------------------------------------------------
# CPU


def test_oracle_matches_reference_tool_golden_rows():
    """Every golden row of the reference tool (5 fields, all 27 predictors, three grids, three
    target modes, rel_eb 1e-1 .. 1e-6): the oracle's BR, H1, RMSE, MAE, PSNR and SAMPLES are the
    same doubles."""
    n = 0
    for case, data, cols in _golden():
        for pred, rows in case["rows"].items():
            for r in rows:
                key = r[0]
                o = O.sweep_run(data, pred, key[0], key[1], key[2] if len(key) > 2 else 0.0, case["targets"])
                got = _cols(o)
                for c, v in zip(cols, r[1:]):
                    assert got[c] == v, (case["name"], pred, key, c, got[c], v)
                n += 1
    assert n == 2007


def test_coefficient_grids_match_golden_keys():
    """The oracle's grids (t = i/32, i/24, and the six-reference grids) equal the keys the tool
    wrote, in order; so do the library's (asz_sweep_coefs, host-side)."""
    from asz_b200 import sweep
    for case, data, cols in _golden():
        ebs = [float(x) for x in case["rel_ebs"].split(",")]
        for pred, rows in case["rows"].items():
            co = O.sweep_coefs(pred, case["six_grid"])
            assert sweep.coefficients(pred, case["six_grid"]) == co
            n = 1 if pred[:4] in ("1d4r", "2d4r") else 2
            assert [r[0] for r in rows] == [[e] + list(c[:n]) for e in ebs for c in co]
    for grid in ("legacy", "augmented", "transition"):
        assert sweep.coefficients("1d6r0_xx0", grid) == O.sweep_coefs("1d6r0_xx0", grid)


@pytest.mark.parametrize("shape", [(12, 12, 12), (13, 17, 12), (20, 14, 31), (12, 25, 16), (16, 16, 13)])
def test_kernel_target_mapping_matches_oracle(shape):
    """The kernel's (line, position) -> (coordinates, stream index) mapping, run on the host, visits
    exactly the oracle's targets in the oracle's order, for all 27 predictors and 3 target modes."""
    from asz_b200 import sweep
    for pred in sweep.predictors("all"):
        for mode in ("legacy", "shared1d", "common"):
            got = sweep.targets(shape, pred, mode)
            exp = O.sweep_targets(shape, pred, mode)
            assert np.array_equal(got, exp), (shape, pred, mode)


def _ref_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libs2_ref.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    L.s2ref_dot.argtypes = [C.c_int, C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_double, C.c_double,
                            C.c_double, C.c_double, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    L.s2ref_h1.argtypes = [C.c_void_p, C.c_uint64]
    L.s2ref_h1.restype = C.c_double
    L.s2ref_grid.argtypes = [C.c_char_p, C.c_void_p, C.c_uint64]
    L.s2ref_grid.restype = C.c_uint64
    L.s2ref_common.argtypes = [C.POINTER(C.c_uint64), C.c_int, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]
    L.s2ref_common.restype = C.c_uint64
    return L


@pytest.mark.skipif(_ref_lib() is None, reason="reference sweep not built (make -C oracle ref)")
def test_oracle_matches_reference_functions():
    """Target by target against the reference's own compress_*_dot, get_H1, six_reference_grid and
    for_each_common_target built with its flags: every QB, the three running sums and H1 are the
    same bits, on random fields and error bounds down to 1e-7."""
    L = _ref_lib()
    rng = np.random.default_rng(8)
    u64 = lambda v: (C.c_uint64 * len(v))(*v)
    for grid in ("legacy", "augmented", "transition"):
        buf = np.empty(256)
        n = L.s2ref_grid(grid.encode(), buf.ctypes.data, 128)
        assert O.sweep_coefs("1d6r1_xx1", grid) == list(zip(buf[0:2 * n:2].tolist(), buf[1:2 * n:2].tolist()))
    for trial in range(6):
        shape = tuple(int(x) for x in rng.integers(12, 22, 3))
        d = _rng_field(rng, shape, rough=trial % 2 == 1)
        mn, mx = float(d.min()), float(d.max())
        for order in range(3):
            cap = int(np.prod(shape))
            co = np.empty((cap, 3), np.uint64)
            vis = C.c_uint64(0)
            cnt = L.s2ref_common(u64(shape), order, co.ctypes.data, cap, C.byref(vis))
            assert cnt == vis.value
            assert np.array_equal(co[:cnt], O.sweep_targets(shape, f"1d4r0_xx{order}", "common"))
        for pred in ("1d4r0_xx1", "1d4r2_xx2", "2d4r02_xx0", "2d4r12_xx1", "1d6r1_xx0", "1d6r2_xx2"):
            rel = float(10 ** rng.uniform(-7, -1))
            mode = ["legacy", "shared1d", "common"][int(rng.integers(0, 3))]
            coords = O.sweep_targets(shape, pred, mode)
            kind = 0 if pred.startswith("1d4r") else 1 if pred.startswith("2d4r") else 2
            n12 = shape[1] * shape[2]
            dist = lambda a: n12 if a == 0 else shape[2] if a == 1 else 1
            dists = u64([dist(int(pred[4])), dist(int(pred[5])) if kind == 1 else 0])
            abs_eb = rel * (mx - mn)
            for c0, c1 in O.sweep_coefs(pred, "augmented")[::5]:
                row, qb = O.sweep_run(d, pred, rel, c0, c1, mode, with_qb=True)
                rq = np.empty(len(coords), np.int64)
                sums = np.empty(3)
                L.s2ref_dot(kind, d.ctypes.data, u64(shape), dists, abs_eb, 1 / (2 * abs_eb), c0, c1,
                            np.ascontiguousarray(coords).ctypes.data, len(coords), rq.ctypes.data, sums.ctypes.data)
                assert np.array_equal(qb, rq), (pred, mode, c0, c1)
                assert [row.mse_sum, row.rmse_sum, row.mae_sum] == sums.tolist(), (pred, mode, c0, c1)
                assert row.h1 == L.s2ref_h1(rq.ctypes.data, len(rq))


def test_cli_argument_errors(tmp_path):
    """Argument checks that run before any device work: the reference's messages and exit 1."""
    inp = tmp_path / "in.f32"
    np.zeros(12 * 12 * 12, np.float32).tofile(inp)
    cases = [
        ([str(inp), "12", "12"], "use --help for arguments"),
        ([str(inp), "12", "12", "12", str(tmp_path / "o"), "3d4r"], "unknown predictor family or stencil"),
        ([str(inp), "12", "12", "12", str(tmp_path / "o"), "1d4r", "1e-3", "dense"],
         "six-reference grid must be legacy, augmented or transition"),
        ([str(inp), "12", "12", "12", str(tmp_path / "o"), "1d4r", "1e-3", "legacy", "all"],
         "target mode must be legacy, shared1d or common"),
        ([str(inp), "12", "12", "12", str(tmp_path / "o"), "1d4r", "1e-3,-1"], "error bounds must be positive and finite"),
        ([str(inp), "12", "11", "12", str(tmp_path / "o"), "1d4r", "1e-3"],
         "invalid dimensions; each dimension must be at least 12"),
        ([str(inp), "12", "12", "13", str(tmp_path / "o"), "1d4r", "1e-3"], "input size does not match float32 dimensions"),
    ]
    for args, msg in cases:
        r = subprocess.run([CLI] + args, capture_output=True, text=True)
        assert r.returncode == 1 and r.stderr.strip() == f"error: {msg}", (args, r.stderr)
    (tmp_path / "p_1d4r1_xx0.csv").write_text("")
    r = subprocess.run([CLI, str(inp), "12", "12", "12", str(tmp_path / "p"), "1d4r1"], capture_output=True, text=True)
    assert r.returncode == 1 and "output already exists" in r.stderr
    r = subprocess.run([CLI, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("usage: s2_many_prediction input dim0 dim1 dim2 output_prefix")


# ---------------------------------------------------------------------------------------------
# GPU


@pytest.mark.gpu
def test_gpu_sweep_matches_golden(gpu_ctx):
    """The CUDA sweep on every golden case: BR, H1 and SAMPLES equal the reference tool's; RMSE, MAE
    and PSNR within 1e-12 relative (sums in another order); the min/max lines too."""
    from asz_b200 import sweep
    n = 0
    for case, data, cols in _golden():
        ebs = [float(x) for x in case["rel_ebs"].split(",")]
        for pred, rows in case["rows"].items():
            got, (mn, mx) = sweep.run(gpu_ctx, data, pred, ebs, case["targets"], case["six_grid"])
            assert case["stdout_head"][1:] == [f"min_val={mn:f}", f"max_val={mx:f}"]
            assert len(got) == len(rows)
            for g, r in zip(got, rows):
                gc = _cols(g)
                assert [g.rel_eb, g.c0] + ([g.c1] if len(r[0]) > 2 else []) == r[0]
                for c, v in zip(cols, r[1:]):
                    if c in EXACT:
                        assert gc[c] == v, (case["name"], pred, r[0], c, gc[c], v)
                    else:
                        assert abs(gc[c] - v) <= SUM_RTOL * abs(v), (case["name"], pred, r[0], c, gc[c], v)
                n += 1
    assert n == 2007


@pytest.mark.gpu
def test_gpu_sweep_matches_oracle_random(gpu_ctx):
    """Random shapes, fields, predictors, grids, target modes and error bounds (1e-1 .. 1e-7, large
    alphabets included): Huffman and zstd sizes, H1 and the sample count are the oracle's exactly,
    the sums within 1e-12 relative; device-resident input gives the same rows."""
    import torch
    from asz_b200 import sweep
    rng = np.random.default_rng(31)
    for trial in range(10):
        shape = tuple(int(x) for x in rng.integers(12, 48, 3))
        d = _rng_field(rng, shape, rough=trial % 3 == 0)
        preds = sweep.predictors("all")
        pred = preds[int(rng.integers(0, len(preds)))]
        mode = ["legacy", "shared1d", "common"][trial % 3]
        grid = ["legacy", "augmented", "transition"][int(rng.integers(0, 3))]
        ebs = sorted(float(10 ** rng.uniform(-7, -1)) for _ in range(2))
        rows, _ = sweep.run(gpu_ctx, d, pred, ebs, mode, grid)
        co = sweep.coefficients(pred, grid)
        assert len(rows) == len(ebs) * len(co)
        for g in rows[:: max(1, len(rows) // 12)]:
            o = O.sweep_run(d, pred, g.rel_eb, g.c0, g.c1, mode)
            assert (g.samples, g.huffman_bytes, g.zstd_bytes) == (o.samples, o.huffman_bytes, o.zstd_bytes), (pred, mode)
            assert (g.br, g.cr, g.h1) == (o.br, o.cr, o.h1)
            for a, b in ((g.mse_sum, o.mse_sum), (g.rmse_sum, o.rmse_sum), (g.mae_sum, o.mae_sum), (g.psnr, o.psnr)):
                assert abs(a - b) <= SUM_RTOL * abs(b), (pred, mode, a, b)
        if trial < 3:
            rows_dev, _ = sweep.run(gpu_ctx, torch.from_numpy(d).cuda(), pred, ebs, mode, grid)
            assert [(r.zstd_bytes, r.h1, r.mse_sum) for r in rows_dev] == [(r.zstd_bytes, r.h1, r.mse_sum) for r in rows]


@pytest.mark.gpu
def test_gpu_sweep_errors(gpu_ctx):
    """A nonfinite value, a constant field and a predictor name the tool does not know are rejected
    with the reference's messages."""
    import asz_b200.api as api
    from asz_b200 import sweep
    d = np.random.default_rng(2).standard_normal((12, 13, 14)).astype(np.float32)
    bad = d.copy()
    bad[3, 4, 5] = np.nan
    with pytest.raises(api.AszError, match="input contains nonfinite values"):
        sweep.run(gpu_ctx, bad, "1d4r0_xx0", [1e-3])
    with pytest.raises(api.AszError, match="constant input"):
        sweep.run(gpu_ctx, np.full((12, 12, 12), 2.5, np.float32), "1d4r0_xx0", [1e-3])
    with pytest.raises(api.AszError, match="unknown predictor"):
        sweep.run(gpu_ctx, d, "1d4r0_xy0", [1e-3])


@pytest.mark.gpu
def test_gpu_cli_matches_reference_output(tmp_path):
    """bin/s2_many_prediction on a golden case prints the reference tool's lines (every row's
    %f figures, computed here from the golden values) and writes one CSV per predictor."""
    case, data, cols = next(c for c in _golden() if c[0]["name"] == "s2_rough_1d4r_shared1d")
    prefix = tmp_path / "run" / "out"
    r = subprocess.run([CLI, os.path.join(GOLDEN, case["name"] + ".f32"), *map(str, case["shape"]), str(prefix),
                        case["family"], case["rel_ebs"], case["six_grid"], case["targets"]],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert lines[:3] == case["stdout_head"]
    exp = []
    for pred, rows in case["rows"].items():
        for row in rows:
            key, br, h1 = row[0], row[1], row[2]
            cr = 32 / br
            exp += [f"rel_eb={key[0]:f}, t={key[1]:f}", f"BR={br:f}, CR={cr:f}", f"H1={h1:f}, H1_cr={32 / h1:f}",
                    f"RMSE={row[3]:f}, MAE={row[4]:f}", f"PSNR={row[5]:f}", ""]
        exp.append(f"predictor={pred}, elapsed_seconds=")
    got = [ln if not ln.startswith("predictor=") else ln[: ln.index("=", 10) + 1] for ln in lines[3:-1]]
    assert got == exp
    assert lines[-1].startswith("total_seconds=")
    for pred, rows in case["rows"].items():
        with open(f"{prefix}_{pred}.csv") as f:
            body = f.read().splitlines()
        assert body[0].startswith("rel_eb,t,BR,H1")
        assert [float(x.split(",")[2]) for x in body[1:]] == [row[1] for row in rows]
