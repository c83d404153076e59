"""ctypes access to the CPU oracle and to the reference binaries compiled from source.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py``, never by the product. ``liboracle()`` loads ``_build/libasz_oracle.so``
(this directory's Makefile). ``ref_binary()`` locates ``_ref/{s1_compress,s1_decompress,ref_dump}``,
built by ``make ref`` from the reference sources where they are present.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class Params(C.Structure):
    _fields_ = [
        ("pivot_eb_ratio", C.c_float), ("eb_ratio", C.c_float), ("slope_ratio", C.c_float),
        ("block_pivot_ratio", C.c_uint64), ("t_precision", C.c_int32),
        ("t_min", C.c_float), ("t_max", C.c_float), ("h1_block_sampling_num", C.c_uint64),
        ("stat_eb_ratio", C.c_float), ("default_slope_invalid_ratio_threshold", C.c_float),
        ("default_slope_fallback", C.c_float), ("default_slope_eb_span", C.c_float),
        ("insufficient_sample_t", C.c_float),
        ("max_layer_num", C.c_uint64), ("full_predictor_search_layer_num", C.c_uint64),
        ("generate_config_sample_stride", C.c_uint64),
        ("predictor_family_suffix_layers", C.c_uint64), ("predictor_family_sample_blocks", C.c_uint64),
        ("predictor_family_sample_point_limit", C.c_uint64), ("predictor_family_sample_fraction_limit", C.c_float),
        ("predictor_family_coarse_probe_block_pivot_ratio", C.c_uint64),
        ("predictor_family_fine_probe_block_pivot_ratio", C.c_uint64),
        ("predictor_family_fine_eb_threshold", C.c_float),
    ]


class _Result(C.Structure):
    _fields_ = [
        ("layer_num", C.c_uint32), ("qb_len", C.POINTER(C.c_uint64)),
        ("qb", C.POINTER(C.POINTER(C.c_int32))), ("t_len", C.c_uint64),
        ("t_int", C.POINTER(C.c_int64)), ("recon", C.POINTER(C.c_float)),
        ("pre_zstd", C.POINTER(C.c_uint8)), ("pre_zstd_len", C.c_uint64),
        ("asz", C.POINTER(C.c_uint8)), ("asz_len", C.c_uint64),
        ("min_val", C.c_float), ("max_val", C.c_float), ("abs_eb", C.c_float),
        ("default_slope", C.c_float), ("t_fallback_count", C.c_uint64),
        ("plan", C.c_char * (64 * 11 + 1)), ("search_layers", C.c_uint32), ("best_dist", C.c_float * 64),
        ("quintic", C.c_int32), ("family_selected", C.c_int32), ("family_fallback", C.c_int32),
        ("fam_suffix_layers", C.c_uint64), ("fam_blocks", C.c_uint64), ("fam_sampled_points", C.c_uint64),
        ("fam_budget", C.c_uint64), ("fam_probe_bpr", C.c_uint64), ("fam_points", C.c_uint64),
        ("fam_cubic_mse", C.c_longdouble), ("fam_quintic_mse", C.c_longdouble), ("fam_cubic_psnr", C.c_longdouble),
        ("fam_quintic_psnr", C.c_longdouble), ("fam_cubic_h1", C.c_longdouble), ("fam_quintic_h1", C.c_longdouble),
        ("fam_score_gain", C.c_longdouble),
    ]


class SweepRow(C.Structure):
    _fields_ = [("c0", C.c_double), ("c1", C.c_double), ("samples", C.c_uint64), ("huffman_bytes", C.c_uint64),
                ("zstd_bytes", C.c_uint64), ("mse_sum", C.c_double), ("rmse_sum", C.c_double), ("mae_sum", C.c_double),
                ("br", C.c_double), ("cr", C.c_double), ("h1", C.c_double), ("h1_cr", C.c_double), ("rmse", C.c_double),
                ("mae", C.c_double), ("psnr", C.c_double)]


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def liboracle():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "_build", "libasz_oracle.so")
        if not os.path.exists(path):
            build_oracle()
        lib = C.CDLL(path)
        lib.aszo_default_params.argtypes = [C.POINTER(Params)]
        lib.aszo_compress.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.c_float, C.POINTER(Params),
                                      C.c_char_p, C.c_int, C.POINTER(_Result), C.c_char_p]
        lib.aszo_compress_with_t.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.c_float, C.POINTER(Params),
                                             C.c_char_p, C.c_int, C.c_void_p, C.c_uint64, C.POINTER(_Result),
                                             C.c_char_p]
        lib.aszo_free_result.argtypes = [C.POINTER(_Result)]
        lib.aszo_grad_samples.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.c_float, C.POINTER(Params), C.c_char_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64),
                                          C.POINTER(C.c_uint64), C.c_char_p]
        lib.aszo_decompress.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64), C.c_float,
                                        C.POINTER(Params), C.c_void_p, C.c_char_p]
        lib.aszo_default_slope.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.c_float, C.c_float,
                                           C.c_float, C.POINTER(Params)]
        lib.aszo_default_slope.restype = C.c_float
        lib.aszo_huffman_encode.argtypes = [C.c_void_p, C.c_uint64, C.c_int, C.c_void_p]
        lib.aszo_huffman_encode.restype = C.c_uint64
        lib.aszo_abmap_order.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]
        lib.aszo_abmap_order.restype = C.c_uint64
        lib.aszo_i64map_order.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p]
        lib.aszo_i64map_order.restype = C.c_uint64
        lib.aszo_h1_psnr.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_float, C.c_float, C.c_float,
                                     C.c_float, C.c_float] + [C.POINTER(C.c_float)] * 4
        lib.aszo_sweep_coefs.argtypes = [C.c_char_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint64]
        lib.aszo_sweep_targets.argtypes = [C.POINTER(C.c_uint64), C.c_char_p, C.c_char_p, C.c_void_p, C.c_uint64]
        lib.aszo_sweep_targets.restype = C.c_uint64
        lib.aszo_sweep_run.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.c_char_p, C.c_char_p, C.c_double,
                                       C.c_float, C.c_float, C.c_double, C.c_double, C.c_void_p, C.c_uint64,
                                       C.POINTER(SweepRow), C.c_char_p]
        lib.aszo_sweep_finish.argtypes = [C.POINTER(SweepRow), C.c_double]
        _LIB = lib
    return _LIB


def default_params(**kw) -> Params:
    p = Params()
    liboracle().aszo_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@dataclass
class Compressed:
    qb: list
    t_int: np.ndarray
    recon: np.ndarray
    pre_zstd: bytes
    asz: bytes
    min_val: float
    max_val: float
    abs_eb: float
    default_slope: float
    t_fallback_count: int
    plan: str = ""
    best_dist: tuple = ()
    quintic: bool = False
    family: dict = None


def _dims(shape):
    return (C.c_uint64 * 3)(*[int(s) for s in shape])


def compress(data: np.ndarray, rel_eb: float, plan: str | None, quintic=False, params: Params | None = None,
             t_int: np.ndarray | None = None) -> Compressed:
    """Compress with `plan`, or run the reference's plan search when plan is None. quintic: a bool,
    or None to run the reference's predictor-family selector. t_int: block-major per-(block, round)
    t codes to use instead of the coefficient selection (needs a plan and a family)."""
    lib = liboracle()
    data = np.ascontiguousarray(data, dtype=np.float32)
    p = params or default_params()
    res = _Result()
    err = C.create_string_buffer(256)
    if t_int is not None:
        t_arr = np.ascontiguousarray(t_int, dtype=np.int64)
        rc = lib.aszo_compress_with_t(data.ctypes.data, _dims(data.shape), C.c_float(rel_eb), C.byref(p),
                                      plan.encode() if plan is not None else None, -1 if quintic is None else int(quintic),
                                      t_arr.ctypes.data, t_arr.size, C.byref(res), err)
    else:
        rc = lib.aszo_compress(data.ctypes.data, _dims(data.shape), C.c_float(rel_eb), C.byref(p),
                               plan.encode() if plan is not None else None, -1 if quintic is None else int(quintic),
                               C.byref(res), err)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    try:
        qb = [np.ctypeslib.as_array(res.qb[i], shape=(res.qb_len[i],)).copy() if res.qb_len[i] else
              np.zeros(0, np.int32) for i in range(res.layer_num + 1)]
        t = np.ctypeslib.as_array(res.t_int, shape=(res.t_len,)).copy() if res.t_len else np.zeros(0, np.int64)
        rec = np.ctypeslib.as_array(res.recon, shape=(data.size,)).copy().reshape(data.shape)
        pre = C.string_at(res.pre_zstd, res.pre_zstd_len)
        asz = C.string_at(res.asz, res.asz_len)
        return Compressed(qb, t, rec, pre, asz, res.min_val, res.max_val, res.abs_eb, res.default_slope,
                          int(res.t_fallback_count), res.plan.decode(),
                          tuple(res.best_dist[i] for i in range(res.search_layers)), bool(res.quintic),
                          {k: getattr(res, k) for k in ("family_selected", "family_fallback", "fam_suffix_layers",
                                                          "fam_blocks", "fam_sampled_points", "fam_budget",
                                                          "fam_probe_bpr", "fam_points", "fam_cubic_mse",
                                                          "fam_quintic_mse", "fam_cubic_psnr", "fam_quintic_psnr",
                                                          "fam_cubic_h1", "fam_quintic_h1", "fam_score_gain")})
    finally:
        lib.aszo_free_result(C.byref(res))


def grad_samples(data: np.ndarray, rel_eb: float, plan: str, params: Params | None = None):
    """(A, B, offsets) of the gradient tuner's open-loop samples, block-major groups."""
    lib = liboracle()
    data = np.ascontiguousarray(data, dtype=np.float32)
    p = params or default_params()
    err = C.create_string_buffer(256)
    g, s = C.c_uint64(), C.c_uint64()
    rc = lib.aszo_grad_samples(data.ctypes.data, _dims(data.shape), C.c_float(rel_eb), C.byref(p), plan.encode(),
                               None, None, None, 0, C.byref(g), C.byref(s), err)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    A = np.empty(s.value, np.float32)
    B = np.empty(s.value, np.float32)
    off = np.empty(g.value + 1, np.uint64)
    rc = lib.aszo_grad_samples(data.ctypes.data, _dims(data.shape), C.c_float(rel_eb), C.byref(p), plan.encode(),
                               A.ctypes.data, B.ctypes.data, off.ctypes.data, s.value, C.byref(g), C.byref(s), err)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return A, B, off


def decompress(asz: bytes, shape, rel_eb: float, params: Params | None = None) -> np.ndarray:
    lib = liboracle()
    p = params or default_params()
    out = np.empty(tuple(shape), dtype=np.float32)
    err = C.create_string_buffer(256)
    buf = C.create_string_buffer(bytes(asz), len(asz))
    rc = lib.aszo_decompress(buf, len(asz), _dims(shape), C.c_float(rel_eb), C.byref(p), out.ctypes.data, err)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return out


def huffman_encode(symbols: np.ndarray) -> bytes:
    lib = liboracle()
    wide = symbols.dtype == np.int64
    s = np.ascontiguousarray(symbols, dtype=np.int64 if wide else np.int32)
    n = lib.aszo_huffman_encode(s.ctypes.data, s.size, int(wide), None)
    out = (C.c_uint8 * n)()
    lib.aszo_huffman_encode(s.ctypes.data, s.size, int(wide), out)
    return bytes(out)


def abmap_order(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, np.int64)
    b = np.ascontiguousarray(b, np.int64)
    out = np.empty(a.size, np.uint64)
    k = liboracle().aszo_abmap_order(a.ctypes.data, b.ctypes.data, a.size, out.ctypes.data)
    return out[:k].astype(np.int64)


def i64map_order(keys: np.ndarray) -> np.ndarray:
    keys = np.ascontiguousarray(keys, np.int64)
    out = np.empty(keys.size, np.uint64)
    k = liboracle().aszo_i64map_order(keys.ctypes.data, keys.size, out.ctypes.data)
    return out[:k].astype(np.int64)


def sweep_coefs(predictor: str, six_grid: str = "legacy"):
    """Coefficient list of a sweep predictor: [(c0, c1), ...]."""
    a, b = np.empty(128), np.empty(128)
    n = liboracle().aszo_sweep_coefs(predictor.encode(), six_grid.encode(), a.ctypes.data, b.ctypes.data, 128)
    if n < 0:
        raise ValueError(predictor)
    return list(zip(a[:n].tolist(), b[:n].tolist()))


def sweep_targets(shape, predictor: str, targets: str = "legacy") -> np.ndarray:
    """(S, 3) uint64 target coordinates in stream order."""
    lib = liboracle()
    n = lib.aszo_sweep_targets(_dims(shape), predictor.encode(), targets.encode(), None, 0)
    out = np.empty((n, 3), np.uint64)
    lib.aszo_sweep_targets(_dims(shape), predictor.encode(), targets.encode(), out.ctypes.data, n)
    return out


def sweep_run(data: np.ndarray, predictor: str, rel_eb: float, c0: float, c1: float = 0.0, targets: str = "legacy",
              with_qb: bool = False):
    """One sweep row on the CPU: SweepRow (and the int64 QB stream when with_qb)."""
    lib = liboracle()
    d = np.ascontiguousarray(data, np.float32)
    mn, mx = float(d.min()), float(d.max())
    cap = int(d.size) if with_qb else 0
    qb = np.empty(cap, np.int64)
    row, err = SweepRow(), C.create_string_buffer(256)
    rc = lib.aszo_sweep_run(d.ctypes.data, _dims(d.shape), predictor.encode(), targets.encode(), rel_eb, mn, mx, c0, c1,
                            qb.ctypes.data if with_qb else None, cap, C.byref(row), err)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return (row, qb[: row.samples]) if with_qb else row


# ---------------------------------------------------------------------------------------------
# The reference compiled from its own sources (oracle/_ref, see the Makefile's `ref` target).

def ref_binary(name: str) -> str | None:
    path = os.path.join(HERE, "_ref", name)
    return path if os.path.exists(path) else None


def read_dump(path: str) -> dict:
    """Parse the `<asz>.dump` written by ref_dump (format in ref_dump.cpp)."""
    with open(path, "rb") as f:
        raw = f.read()
    assert raw[:8] == b"ASZDUMP1"
    off = 8

    def u64():
        nonlocal off
        v = struct.unpack_from("<Q", raw, off)[0]
        off += 8
        return v

    nstreams = u64()
    qb = []
    for _ in range(nstreams):
        n = u64()
        qb.append(np.frombuffer(raw, np.int32, n, off).copy())
        off += 4 * n
    n = u64()
    t = np.frombuffer(raw, np.int64, n, off).copy()
    off += 8 * n
    n = u64()
    rec = np.frombuffer(raw, np.float32, n, off).copy()
    off += 4 * n
    mn, mx, abs_eb, slope = struct.unpack_from("<ffff", raw, off)
    off += 16
    quintic = raw[off]
    off += 1
    n = u64()
    plan = raw[off:off + n].decode()
    return dict(qb=qb, t_int=t, recon=rec, min_val=mn, max_val=mx, abs_eb=abs_eb, default_slope=slope,
                quintic=bool(quintic), plan=plan)


def run_reference_compress(data: np.ndarray, rel_eb: float, workdir: str, plan: str | None = None,
                           family: str | None = None, extra=(), dump: bool = True, binary: str | None = None):
    """Run the reference compressor (ref_dump or s1_compress) on `data`; returns (asz bytes, dump, stdout)."""
    exe = binary or ref_binary("ref_dump" if dump else "s1_compress")
    if exe is None:
        raise FileNotFoundError("reference binaries not built (make -C oracle ref)")
    inp = os.path.join(workdir, "in.f32")
    out = os.path.join(workdir, "out.asz")
    np.ascontiguousarray(data, np.float32).tofile(inp)
    argv = [exe, "-i", inp, "-z", out, "-3", *[str(s) for s in data.shape], "-M", "REL", repr(float(rel_eb))]
    if plan:
        argv += ["--predictor-plan", plan]
    if family:
        argv += ["--predictor-family", family]
    argv += list(extra)
    r = subprocess.run(argv, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference compressor failed: {r.stderr.strip()}")
    with open(out, "rb") as f:
        asz = f.read()
    d = read_dump(out + ".dump") if dump and os.path.exists(out + ".dump") else None
    return asz, d, r.stdout


def run_reference_decompress(asz: bytes, shape, rel_eb: float, workdir: str, extra=()) -> np.ndarray:
    exe = ref_binary("s1_decompress")
    if exe is None:
        raise FileNotFoundError("reference binaries not built (make -C oracle ref)")
    z = os.path.join(workdir, "d.asz")
    o = os.path.join(workdir, "d.out")
    with open(z, "wb") as f:
        f.write(asz)
    argv = [exe, "-z", z, "-o", o, "-3", *[str(s) for s in shape], "-M", "REL", repr(float(rel_eb)), *extra]
    r = subprocess.run(argv, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference decompressor failed: {r.stderr.strip()}")
    return np.fromfile(o, np.float32).reshape(tuple(shape))
