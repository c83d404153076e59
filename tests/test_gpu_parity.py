"""Parity of the CUDA path with the reference: golden vectors written by the reference binary,
randomised cases against the CPU oracle (QB streams, t codes, reconstruction, stream bytes), the
drop-in CLI, device-resident inputs, and corrupt-stream handling."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, golden_cases, load_golden

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "asz_b200", "bin")


def _params(api, **kw):
    return api.default_params(**kw)


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c["name"])
def test_golden_compress_and_decompress(gpu_ctx, case):
    import asz_b200.api as api
    data, blob, out = load_golden(case)
    p = _params(api, block_pivot_ratio=case["block_pivot_ratio"])
    got, rep = gpu_ctx.compress(data, case["rel_eb"], case["plan"], case["family"], p)
    assert got == blob
    rec = gpu_ctx.debug_recon().reshape(data.shape)
    assert np.array_equal(rec.view(np.uint32), out.view(np.uint32))
    dec, _ = gpu_ctx.decompress(blob, data.shape, case["rel_eb"], _params(api, block_pivot_ratio=case["block_pivot_ratio"]))
    assert np.array_equal(dec.view(np.uint32), out.view(np.uint32))


def _check_against_oracle(ctx, data, eb, plan, family, bpr):
    import asz_b200.api as api
    p = api.default_params(block_pivot_ratio=bpr)
    blob, rep = ctx.compress(data, eb, plan, family, p)
    o = O.compress(data, eb, plan, family == "quintic", O.default_params(block_pivot_ratio=bpr))
    assert rep.default_slope == np.float32(o.default_slope) or (np.isnan(rep.default_slope) and np.isnan(o.default_slope))
    assert np.array_equal(ctx.debug_t(), o.t_int)
    for s, q in enumerate(o.qb):
        assert np.array_equal(ctx.debug_qb(s), q), f"QB stream {s}"
    assert np.array_equal(ctx.debug_recon().view(np.uint32), o.recon.ravel().view(np.uint32))
    assert ctx.debug_pre_zstd() == o.pre_zstd
    assert blob == o.asz
    dec, _ = ctx.decompress(blob, data.shape, eb, api.default_params(block_pivot_ratio=bpr))
    assert np.array_equal(dec.view(np.uint32), o.recon.view(np.uint32))
    return rep


@pytest.mark.parametrize("mode", [0, 1], ids=["fast+exact", "exact-only"])
def test_random_cases_against_oracle(gpu_ctx, mode):
    from asz_b200 import fields
    gpu_ctx.set_tsel_mode(mode)
    rng = np.random.default_rng(99 + mode)
    orders = ["120", "021", "012"]
    for i in range(40):
        shape = tuple(int(x) for x in rng.integers(7, 48, size=3))
        f = fields.grf_field(shape, rng.uniform(1.2, 5), rng)
        kind = i % 4
        if kind == 1:
            f[: shape[0] // 3] = 0.0
        elif kind == 2:
            f = np.round(f * 4) / 4
        elif kind == 3:
            f = f + 10 * np.tanh((np.arange(shape[2]) - shape[2] / 2) / 2)[None, None, :]
        f = f.astype(np.float32)
        plan = ",".join(f"cubic{rng.integers(0, 3)}_{orders[rng.integers(0, 3)]}" for _ in range(int(rng.integers(1, 10))))
        family = ["cubic", "quintic"][int(rng.integers(0, 2))]
        eb = float(10 ** rng.uniform(-5, -1.5))
        bpr = int(rng.integers(1, 6))
        _check_against_oracle(gpu_ctx, f, eb, plan, family, bpr)
    gpu_ctx.set_tsel_mode(0)


@pytest.mark.parametrize("family", ["cubic", "quintic"])
def test_c2_like_128_cubic2_plan(gpu_ctx, family):
    """The headline plan shape (cubic2_012 on every level, launcher block ratio 3) at 128^3."""
    from asz_b200 import fields
    f = fields.c2_field(shape=(128, 128, 128))
    rep = _check_against_oracle(gpu_ctx, f, 1e-3, ",".join(["cubic2_012"] * 7), family, 3)
    assert rep.t_fallback_count > 0


@pytest.mark.parametrize("mode", [2, 0], ids=["fused", "per-round"])
def test_axis2_plans_fused_rounds(gpu_ctx, mode):
    """Plans with every round along axis 2, with all rounds fused per column of lines (mode 2) and
    one launch per round (mode 0): random shapes, block ratios (1 to 64 blocks along
    axis 2), families and error bounds, with noise fields whose groups the fast path hands to the
    exact path part-way through a column."""
    from asz_b200 import fields
    gpu_ctx.set_tsel_mode(mode)
    rng = np.random.default_rng(2024)
    handed_off = 0
    for i in range(16):
        shape = (int(rng.integers(7, 30)), int(rng.integers(7, 30)), int(rng.integers(16, 400)))
        if i % 4 == 3:
            f = rng.random(shape).astype(np.float32)
            eb = float(10 ** rng.uniform(-5, -4))
        else:
            f = fields.grf_field(shape, rng.uniform(1.2, 5), rng).astype(np.float32)
            eb = float(10 ** rng.uniform(-5, -1.5))
        layers = int(rng.integers(1, 9))
        plan = ",".join(f"cubic2_{['120', '021', '012'][int(rng.integers(0, 3))]}" for _ in range(layers))
        family = ["cubic", "quintic"][i % 2]
        bpr = int(rng.integers(1, 6))
        rep = _check_against_oracle(gpu_ctx, f, eb, plan, family, bpr)
        handed_off += rep.exact_groups
    gpu_ctx.set_tsel_mode(0)
    assert handed_off > 0


def test_plan_search_against_oracle(gpu_ctx):
    """No plan given: the device plan search picks the reference's plan (checked with the oracle's
    restatement), and the whole compression then matches."""
    import asz_b200.api as api
    from asz_b200 import fields
    rng = np.random.default_rng(77)
    for i in range(12):
        shape = tuple(int(x) for x in rng.integers(7, 48, size=3))
        f = fields.grf_field(shape, rng.uniform(1.5, 5), rng).astype(np.float32)
        if i % 3 == 1:
            f[: shape[0] // 3] = 0.0
        eb = float(10 ** rng.uniform(-5, -1.5))
        family = ["cubic", "quintic"][int(rng.integers(0, 2))]
        bpr = int(rng.integers(1, 6))
        o = O.compress(f, eb, None, family == "quintic", O.default_params(block_pivot_ratio=bpr))
        blob, rep = gpu_ctx.compress(f, eb, None, family, api.default_params(block_pivot_ratio=bpr))
        assert rep.plan.decode() == o.plan
        assert [rep.plan_best_dist[k] for k in range(rep.plan_search_layers)] == list(o.best_dist)
        assert blob == o.asz


def test_family_selection_against_oracle(gpu_ctx):
    """No family given: the device-run probes make the reference's choice (via the oracle's
    restatement) with the same long-double figures, on fixed and searched plans."""
    import asz_b200.api as api
    from asz_b200 import fields
    rng = np.random.default_rng(131)
    orders = ["120", "021", "012"]
    families = set()
    for i in range(16):
        shape = tuple(int(x) for x in rng.integers(7, 60, size=3))
        f = fields.grf_field(shape, rng.uniform(1.5, 5), rng).astype(np.float32)
        eb = float(10 ** rng.uniform(-5, -1.5))
        plan = None if i % 4 == 0 else ",".join(
            f"cubic{rng.integers(0, 3)}_{orders[rng.integers(0, 3)]}" for _ in range(int(rng.integers(1, 10))))
        bpr = int(rng.integers(1, 6))
        try:
            o = O.compress(f, eb, plan, None, O.default_params(block_pivot_ratio=bpr))
        except RuntimeError as e:
            with pytest.raises(api.AszError, match="no target points"):
                gpu_ctx.compress(f, eb, plan, "auto", api.default_params(block_pivot_ratio=bpr))
            assert "no target points" in str(e)
            continue
        blob, rep = gpu_ctx.compress(f, eb, plan, "auto", api.default_params(block_pivot_ratio=bpr))
        assert bool(rep.quintic) == o.quintic
        families.add(o.quintic)
        for k in ("fam_cubic_mse", "fam_quintic_mse", "fam_cubic_psnr", "fam_quintic_psnr", "fam_cubic_h1",
                  "fam_quintic_h1", "fam_score_gain"):
            assert getattr(rep, k) == o.family[k], k
        assert blob == o.asz


def test_plan_search_c1_like(gpu_ctx):
    """A C1-shaped field (smaller depth) through the plan search, against the oracle."""
    import asz_b200.api as api
    from asz_b200 import fields
    f = fields.c1_field(seed=3, shape=(24, 120, 100))
    o = O.compress(f, 1e-3, None, False, O.default_params(block_pivot_ratio=3))
    blob, rep = gpu_ctx.compress(f, 1e-3, None, "cubic", api.default_params(block_pivot_ratio=3))
    assert rep.plan.decode() == o.plan
    assert blob == o.asz


@pytest.mark.parametrize("rel_eb,path", [(1e-4, "windows"), (2e-5, "exact")])
def test_wide_bin_ranges(gpu_ctx, rel_eb, path):
    """White noise at a small error bound: the quantised errors of many (block, round) groups span
    more than the fast path's histogram window, so they are counted window by window (or, when
    too spread, handed to the exact path)."""
    rng = np.random.default_rng(5)
    f = rng.random((24, 24, 384)).astype(np.float32)
    rep = _check_against_oracle(gpu_ctx, f, rel_eb, ",".join(["cubic2_012"] * 6), "cubic", 3)
    if path == "windows":
        assert rep.wide_groups > 0
    else:
        assert rep.exact_window > 0


def test_device_resident_input(gpu_ctx):
    import torch

    import asz_b200.api as api
    case = golden_cases()[0]
    data, blob, out = load_golden(case)
    x = torch.from_numpy(data).cuda()
    got, _ = gpu_ctx.compress(x, case["rel_eb"], case["plan"], case["family"],
                              api.default_params(block_pivot_ratio=case["block_pivot_ratio"]))
    assert got == blob
    y = torch.empty_like(x)
    gpu_ctx.decompress(blob, data.shape, case["rel_eb"], api.default_params(block_pivot_ratio=case["block_pivot_ratio"]),
                       out=y)
    torch.cuda.synchronize()
    assert np.array_equal(y.cpu().numpy().view(np.uint32), out.view(np.uint32))


def test_device_input_not_16_byte_aligned(gpu_ctx):
    """The finest round along axis 2 stages whole lines with 16-byte loads when the input allows; a
    device input 4 bytes past a 16-byte boundary takes the per-target kernel. Both match the oracle."""
    import torch

    import asz_b200.api as api
    from asz_b200 import fields
    f = fields.c2_field(seed=9, shape=(24, 32, 64))
    plan = ",".join(["cubic2_012"] * 5)
    o = O.compress(f, 1e-3, plan, False, O.default_params(block_pivot_ratio=3))
    aligned = torch.from_numpy(f).cuda()
    flat = torch.empty(f.size + 1, dtype=torch.float32, device="cuda")
    flat[1:].copy_(aligned.view(-1))
    shifted = flat[1:].view(f.shape)
    assert aligned.data_ptr() % 16 == 0 and shifted.data_ptr() % 16 == 4
    for x in (aligned, shifted):
        blob, _ = gpu_ctx.compress(x, 1e-3, plan, "cubic", api.default_params(block_pivot_ratio=3))
        assert blob == o.asz
        assert np.array_equal(gpu_ctx.debug_recon().view(np.uint32), o.recon.ravel().view(np.uint32))


@pytest.mark.parametrize("shape", [(9, 7, 1024), (7, 7, 4096)], ids=["n2_1024", "n2_4096"])
@pytest.mark.parametrize("family", ["cubic", "quintic"])
def test_long_lines_against_oracle(gpu_ctx, shape, family):
    """Lines of 1024 and 4096 points: the finest round's line-staging kernel with more than 48 KB of
    shared memory per CTA (eight and three warps)."""
    from asz_b200 import fields
    f = fields.c2_field(seed=11, shape=shape)
    _check_against_oracle(gpu_ctx, f, 1e-3, ",".join(["cubic2_012"] * 4), family, 3)


@pytest.mark.parametrize("case", golden_cases()[:3], ids=lambda c: c["name"])
def test_cli_drop_in(case):
    data, blob, out = load_golden(case)
    dims = [str(s) for s in data.shape]
    with tempfile.TemporaryDirectory() as wd:
        inp, z, o = os.path.join(wd, "in.f32"), os.path.join(wd, "x.asz"), os.path.join(wd, "x.out")
        data.tofile(inp)
        flags = ["--block-pivot-ratio", str(case["block_pivot_ratio"])]
        r = subprocess.run([os.path.join(BIN, "s1_compress"), "-f", "-i", inp, "-z", z, "-3", *dims, "-M", "REL",
                            repr(case["rel_eb"]), "--predictor-plan", case["plan"], "--predictor-family", case["family"],
                            *flags], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert open(z, "rb").read() == blob
        for line in ("Compression time:", "CR: ", "max_err=", "predictor_vec={", "Default slope statistics:"):
            assert line in r.stdout
        r = subprocess.run([os.path.join(BIN, "s1_decompress"), "-z", z, "-o", o, "-3", *dims, "-M", "REL",
                            repr(case["rel_eb"]), *flags], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert np.array_equal(np.fromfile(o, np.float32), out.ravel())
        assert "Decompression time:" in r.stdout and "CR= " in r.stdout


def test_cli_plan_search():
    """s1_compress without --predictor-plan: the searched plan's .asz (checked with the oracle) and the
    plan-search stdout lines."""
    case = golden_cases()[0]
    data, _, _ = load_golden(case)
    dims = [str(s) for s in data.shape]
    bpr = case["block_pivot_ratio"]
    want = O.compress(data, case["rel_eb"], None, case["family"] == "quintic", O.default_params(block_pivot_ratio=bpr))
    with tempfile.TemporaryDirectory() as wd:
        inp, z = os.path.join(wd, "in.f32"), os.path.join(wd, "x.asz")
        data.tofile(inp)
        r = subprocess.run([os.path.join(BIN, "s1_compress"), "-f", "-i", inp, "-z", z, "-3", *dims, "-M", "REL",
                            repr(case["rel_eb"]), "--predictor-family", case["family"], "--block-pivot-ratio", str(bpr)],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert open(z, "rb").read() == want.asz
        for line in ("best_layer_predictor=", "Generate config breakdown: statistics=", "Generate config time:"):
            assert line in r.stdout


def test_cli_fully_automatic():
    """s1_compress with neither a plan nor a family (the launcher's default), against the oracle."""
    from asz_b200 import fields
    f = fields.c1_field(seed=5, shape=(20, 64, 60))
    want = O.compress(f, 1e-3, None, None, O.default_params(block_pivot_ratio=3))
    with tempfile.TemporaryDirectory() as wd:
        inp, z = os.path.join(wd, "in.f32"), os.path.join(wd, "x.asz")
        f.tofile(inp)
        r = subprocess.run([os.path.join(BIN, "s1_compress"), "-f", "-i", inp, "-z", z, "-3", *[str(s) for s in f.shape],
                            "-M", "REL", "0.001", "--block-pivot-ratio", "3"], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert open(z, "rb").read() == want.asz
        assert "Predictor family selection: selector=h1" in r.stdout
        assert "Predictor family selection time:" in r.stdout


def test_corrupt_streams_fail_cleanly(gpu_ctx):
    import asz_b200.api as api
    case = golden_cases()[0]
    data, blob, out = load_golden(case)
    p = api.default_params(block_pivot_ratio=case["block_pivot_ratio"])
    for bad in (blob[: len(blob) // 2], b"\x00" * 16, blob[:-3]):
        with pytest.raises(api.AszError):
            gpu_ctx.decompress(bad, data.shape, case["rel_eb"], p)
    # A well-formed stream decoded with the wrong block ratio still must not fault the device.
    raw = O.compress(data, case["rel_eb"], case["plan"], case["family"] == "quintic",
                     O.default_params(block_pivot_ratio=case["block_pivot_ratio"])).pre_zstd
    assert len(raw) > 0
    dec, _ = gpu_ctx.decompress(blob, data.shape, case["rel_eb"], p)
    assert np.array_equal(dec.view(np.uint32), out.view(np.uint32))


def _zstd3(raw: bytes) -> bytes:
    import ctypes as C
    z = C.CDLL("libzstd.so.1")
    z.ZSTD_compressBound.restype = C.c_size_t
    z.ZSTD_compressBound.argtypes = [C.c_size_t]
    z.ZSTD_compress.restype = C.c_size_t
    z.ZSTD_compress.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_int]
    cap = z.ZSTD_compressBound(len(raw))
    buf = C.create_string_buffer(cap)
    n = z.ZSTD_compress(buf, cap, raw, len(raw), 3)
    return buf.raw[:n]


def test_corrupt_payload_bits(gpu_ctx):
    """Bit flips inside the Huffman payloads (re-wrapped in a valid zstd frame): the decoder either
    reports a corrupt stream or decodes some other valid stream, never faults, and the context
    keeps working."""
    import asz_b200.api as api
    case = golden_cases()[0]
    data, blob, out = load_golden(case)
    p = api.default_params(block_pivot_ratio=case["block_pivot_ratio"])
    raw = O.compress(data, case["rel_eb"], case["plan"], case["family"] == "quintic",
                     O.default_params(block_pivot_ratio=case["block_pivot_ratio"])).pre_zstd
    rng = np.random.default_rng(3)
    errors = 0
    for _ in range(24):
        b = bytearray(raw)
        for _ in range(int(rng.integers(1, 4))):
            i = int(rng.integers(len(b) // 2, len(b)))
            b[i] ^= 1 << int(rng.integers(0, 8))
        try:
            gpu_ctx.decompress(_zstd3(bytes(b)), data.shape, case["rel_eb"], p)
        except api.AszError:
            errors += 1
    assert errors > 0
    dec, _ = gpu_ctx.decompress(blob, data.shape, case["rel_eb"], p)
    assert np.array_equal(dec.view(np.uint32), out.view(np.uint32))

