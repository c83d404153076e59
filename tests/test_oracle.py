"""The CPU oracle against the reference: committed golden vectors, the reference binaries built
from source (when present), and known-answer checks of the Huffman layout and hash-table order."""
import os
import struct
import tempfile

import numpy as np
import pytest

import oracle as O
from conftest import golden_cases, load_golden


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c["name"])
def test_oracle_matches_golden(case):
    data, blob, out = load_golden(case)
    p = O.default_params(block_pivot_ratio=case["block_pivot_ratio"])
    c = O.compress(data, case["rel_eb"], case["plan"], case["family"] == "quintic", p)
    assert c.asz == blob
    assert np.array_equal(c.recon.view(np.uint32), out.view(np.uint32))
    dec = O.decompress(blob, data.shape, case["rel_eb"], p)
    assert np.array_equal(dec.view(np.uint32), out.view(np.uint32))
    err = np.abs(out.astype(np.float64) - data.astype(np.float64)).max()
    assert err <= 1.01 * c.abs_eb


def _ref_available():
    return O.ref_binary("ref_dump") is not None and O.ref_binary("s1_decompress") is not None


@pytest.mark.skipif(not _ref_available(), reason="reference binaries not built (make -C oracle ref)")
def test_oracle_matches_reference_binary_random():
    from asz_b200 import fields
    rng = np.random.default_rng(2024)
    orders = ["120", "021", "012"]
    for _ in range(25):
        shape = tuple(int(x) for x in rng.integers(7, 40, size=3))
        f = fields.grf_field(shape, rng.uniform(1.5, 5), rng)
        if rng.random() < 0.3:
            f[: shape[0] // 3] = 0.0
        f = f.astype(np.float32)
        plan = ",".join(f"cubic{rng.integers(0, 3)}_{orders[rng.integers(0, 3)]}" for _ in range(int(rng.integers(1, 8))))
        fam = ["cubic", "quintic"][int(rng.integers(0, 2))]
        eb = float(10 ** rng.uniform(-5, -1.5))
        bpr = int(rng.integers(1, 6))
        p = O.default_params(block_pivot_ratio=bpr)
        with tempfile.TemporaryDirectory() as wd:
            asz, d, _ = O.run_reference_compress(f, eb, wd, plan=plan, family=fam,
                                                 extra=["--block-pivot-ratio", str(bpr)])
            c = O.compress(f, eb, plan, fam == "quintic", p)
            assert c.asz == asz
            assert np.array_equal(c.t_int, d["t_int"])
            for a, b in zip(c.qb, d["qb"]):
                assert np.array_equal(a, b)
            assert np.array_equal(c.recon.view(np.uint32).ravel(), d["recon"].view(np.uint32))
            dec = O.run_reference_decompress(asz, shape, eb, wd, extra=["--block-pivot-ratio", str(bpr)])
            assert np.array_equal(O.decompress(asz, shape, eb, p).view(np.uint32), dec.view(np.uint32))


@pytest.mark.skipif(not _ref_available(), reason="reference binaries not built (make -C oracle ref)")
def test_oracle_plan_search_matches_reference_binary():
    """The plan search (no --predictor-plan): the searched plan and the .asz bytes."""
    import re

    from asz_b200 import fields
    rng = np.random.default_rng(4242)
    for _ in range(10):
        shape = tuple(int(x) for x in rng.integers(7, 40, size=3))
        f = fields.grf_field(shape, rng.uniform(1.5, 5), rng).astype(np.float32)
        eb = float(10 ** rng.uniform(-5, -1.5))
        fam = ["cubic", "quintic"][int(rng.integers(0, 2))]
        bpr = int(rng.integers(1, 6))
        with tempfile.TemporaryDirectory() as wd:
            asz, _, out = O.run_reference_compress(f, eb, wd, plan=None, family=fam,
                                                   extra=["--block-pivot-ratio", str(bpr)], dump=False)
        c = O.compress(f, eb, None, fam == "quintic", O.default_params(block_pivot_ratio=bpr))
        ref_plan = re.search(r'predictor_vec=\{([^}]*)\}', out).group(1).replace('"', '')
        assert c.plan == ref_plan
        assert c.asz == asz
        ref_dists = [float(x) for x in re.findall(r"best_layer_predictor=cubic\d_\d+, best_dist=([-0-9.e+]+)", out)]
        assert np.allclose(ref_dists, c.best_dist, rtol=0, atol=1e-6)


@pytest.mark.skipif(not _ref_available(), reason="reference binaries not built (make -C oracle ref)")
def test_oracle_family_selection_matches_reference_binary():
    """No --predictor-family: the selector's choice, its printed score, and the .asz bytes (the
    reference's own error when no target point is sampled)."""
    import re

    from asz_b200 import fields
    rng = np.random.default_rng(31)
    orders = ["120", "021", "012"]
    seen = set()
    for i in range(14):
        shape = tuple(int(x) for x in rng.integers(7, 60, size=3))
        f = fields.grf_field(shape, rng.uniform(1.5, 5), rng).astype(np.float32)
        eb = float(10 ** rng.uniform(-5, -1.5))
        plan = None if i % 4 == 0 else ",".join(
            f"cubic{rng.integers(0, 3)}_{orders[rng.integers(0, 3)]}" for _ in range(int(rng.integers(1, 10))))
        bpr = int(rng.integers(1, 6))
        ref_err = ora_err = None
        with tempfile.TemporaryDirectory() as wd:
            try:
                asz, _, out = O.run_reference_compress(f, eb, wd, plan=plan, family=None,
                                                       extra=["--block-pivot-ratio", str(bpr)], dump=False)
            except RuntimeError as e:
                ref_err = str(e).split("error: ")[-1]
        try:
            c = O.compress(f, eb, plan, None, O.default_params(block_pivot_ratio=bpr))
        except RuntimeError as e:
            ora_err = str(e)
        assert ref_err == ora_err
        if ref_err:
            continue
        line = [l for l in out.splitlines() if l.startswith("Predictor family selection:")][0]
        assert (re.search(r"family=(\w+)", line).group(1) == "quintic") == c.quintic
        seen.add(c.quintic)
        m = re.search(r"six_score_gain=([-0-9.e+]+)", line)
        if m:
            assert f"{float(c.family['fam_score_gain']):.12e}" == f"{float(m.group(1)):.12e}"
        assert c.asz == asz


@pytest.mark.skipif(not _ref_available(), reason="reference binaries not built (make -C oracle ref)")
def test_given_t_tables_decode_with_reference():
    """Streams compressed with a caller's t table (any code on the t grid in [t_min, t_max], as the
    gradient tuner writes) decode with the reference's own decompressor to the oracle's
    reconstruction, and a table equal to the selection's reproduces the selection's bytes."""
    from asz_b200 import fields
    rng = np.random.default_rng(808)
    for i in range(6):
        shape = tuple(int(x) for x in rng.integers(7, 40, size=3))
        f = fields.grf_field(shape, rng.uniform(1.5, 5), rng).astype(np.float32)
        eb = float(10 ** rng.uniform(-4, -2))
        plan = ",".join(f"cubic{rng.integers(0, 3)}_012" for _ in range(int(rng.integers(1, 7))))
        bpr = int(rng.integers(1, 5))
        p = O.default_params(block_pivot_ratio=bpr)
        quintic = bool(i % 2)
        sel = O.compress(f, eb, plan, quintic, p)
        assert O.compress(f, eb, plan, quintic, p, t_int=sel.t_int).asz == sel.asz
        t = rng.integers(2, 13, size=sel.t_int.shape).astype(np.int64)
        c = O.compress(f, eb, plan, quintic, p, t_int=t)
        assert np.array_equal(c.t_int, t)
        with tempfile.TemporaryDirectory() as wd:
            dec = O.run_reference_decompress(c.asz, shape, eb, wd, extra=["--block-pivot-ratio", str(bpr)])
        assert np.array_equal(dec.view(np.uint32), c.recon.view(np.uint32))
        assert np.abs(dec.astype(np.float64) - f).max() <= 1.01 * c.abs_eb


def test_huffman_known_answer():
    # Symbols [0,0,1]: heap pops leaf 1 (freq 1) then leaf 0 (freq 2) -> codes 1:'0', 0:'1'.
    enc = O.huffman_encode(np.array([0, 0, 1], np.int32))
    hdr = bytes([1]) + struct.pack("<q", 0) + struct.pack(">Q", 2) + struct.pack(">Q", 2)
    tree = bytes([0b01110])                     # preorder: internal, leaf(1), leaf(0)
    lenw = struct.pack(">Q", 3 ^ 0x1234ABCD)
    payload = bytes([0b011])                    # LSB-first: 1, 1, 0
    assert enc == hdr + tree + lenw + payload
    # A single symbol stores only the masked count (huffman.hpp:342-347).
    enc1 = O.huffman_encode(np.array([7, 7, 7, 7], np.int32))
    assert enc1 == bytes([0x41]) + struct.pack("<q", 7) + struct.pack(">Q", 1) + struct.pack(">Q", 1) + \
        struct.pack(">Q", 4 ^ 0x1234ABCD)


# libstdc++ growth schedule (bucket counts after the k-th insertion), as the kernels use it.
SCHED = [(1, 13), (14, 29), (30, 59), (60, 127), (128, 257), (258, 541), (542, 1109), (1110, 2357),
         (2358, 5087), (5088, 10273)]


def _stage_order(seq, hashes, beta):
    created = {}
    for t, e in enumerate(seq):
        created.setdefault(hashes[e] % beta, t)
    return [e for _, _, e in sorted((-created[hashes[e] % beta], -t, e) for t, e in enumerate(seq))]


def _model(hashes):
    order = []
    pts = [(r, b) for r, b in SCHED if r <= len(hashes)]
    for i, (r, beta) in enumerate(pts):
        end = pts[i + 1][0] - 1 if i + 1 < len(pts) else len(hashes)
        order = _stage_order(order + list(range(r - 1, end)), hashes, beta)
    return order


def test_hashtable_order_model():
    """Iteration order of the reference's unordered_maps follows bucket-run creation order."""
    rng = np.random.default_rng(7)
    M = (1 << 64) - 1
    for trial in range(300):
        n = int(rng.integers(1, 1500))
        span = int(rng.integers(1, 50))
        a = rng.integers(-span, span + 1, size=n)
        b = rng.integers(-span, span + 1, size=n)
        ref = list(O.abmap_order(a, b))
        seen, firsts = set(), []
        for i, key in enumerate(zip(a.tolist(), b.tolist())):
            if key not in seen:
                seen.add(key)
                firsts.append(i)
        h = [((int(a[i]) * 1145141919810 + int(b[i])) & M) for i in firsts]
        assert ref == [firsts[e] for e in _model(h)]
        k = rng.integers(-3 * span, 3 * span + 1, size=n)
        refq = list(O.i64map_order(k))
        seen, fq = set(), []
        for i, x in enumerate(k.tolist()):
            if x not in seen:
                seen.add(x)
                fq.append(i)
        assert refq == [fq[e] for e in _model([int(k[i]) & M for i in fq])]


def test_device_hashorder_emulation_matches_container():
    """The ListSim code the kernels run, executed on the host, against std::unordered_map."""
    import ctypes as C

    import asz_b200.api as api
    L = api.lib()
    L.asz_check_hashorder.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_void_p]
    L.asz_check_hashorder.restype = C.c_int64
    rng = np.random.default_rng(17)
    for trial in range(400):
        n = int(rng.integers(1, 6000 if trial % 50 == 0 else 1500))
        span = int(rng.integers(1, 80))
        a = rng.integers(-span, span + 1, size=n).astype(np.int64)
        b = rng.integers(-span, span + 1, size=n).astype(np.int64)
        if trial % 4 == 0:
            a = rng.integers(-2**40, 2**40, size=n).astype(np.int64)
        out = np.empty(n, np.uint64)
        m = L.asz_check_hashorder(a.ctypes.data, b.ctypes.data, n, 1, out.ctypes.data)
        assert m >= 0
        assert np.array_equal(out[:m].astype(np.int64), O.abmap_order(a, b))
        m = L.asz_check_hashorder(a.ctypes.data, None, n, 0, out.ctypes.data)
        assert m >= 0
        assert np.array_equal(out[:m].astype(np.int64), O.i64map_order(a))
