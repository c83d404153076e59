"""The prediction sweep: GPU form of the reference's study tool s2_many_prediction
(c_codes/s2_many_prediction.cpp), over the C ABI (asz_sweep in include/asz_b200.h).

    rows = sweep.run(ctx, field, "1d6r2_xx2", [1e-3, 1e-4], targets="common", six_grid="augmented")
    for r in rows: r.br, r.h1, r.rmse, r.mae, r.psnr, r.samples

Predictors are "1d4r<axis>_xx<order>", "2d4r<axes>_xx<order>" (axes 01, 02, 12) and
"1d6r<axis>_xx<order>"; ``predictors(family)`` lists them the way the tool's family argument
does. The command-line front end with the tool's arguments and output is bin/s2_many_prediction.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import api

STENCILS = ("1d4r0", "1d4r1", "1d4r2", "2d4r01", "2d4r02", "2d4r12", "1d6r0", "1d6r1", "1d6r2")


class SweepRow(C.Structure):
    _fields_ = [("rel_eb", C.c_double), ("c0", C.c_double), ("c1", C.c_double), ("samples", C.c_uint64),
                ("huffman_bytes", C.c_uint64), ("zstd_bytes", C.c_uint64), ("mse_sum", C.c_double),
                ("rmse_sum", C.c_double), ("mae_sum", C.c_double), ("br", C.c_double), ("cr", C.c_double),
                ("h1", C.c_double), ("h1_cr", C.c_double), ("rmse", C.c_double), ("mae", C.c_double),
                ("psnr", C.c_double), ("encode_seconds", C.c_double)]


def _bind(L):
    if getattr(L, "_sweep_bound", False):
        return L
    L.asz_sweep_coefs.argtypes = [C.c_char_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]
    L.asz_sweep_targets.argtypes = [C.POINTER(C.c_uint64), C.c_char_p, C.c_char_p, C.c_void_p, C.c_uint64,
                                    C.POINTER(C.c_uint64)]
    L.asz_sweep.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.c_char_p, C.c_char_p, C.c_char_p,
                            C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64), C.c_void_p]
    L._sweep_bound = True
    return L


def predictors(family: str = "all"):
    """Predictor names for a family-or-stencil argument (s2_many_prediction.cpp:547-553)."""
    if family != "all" and family not in ("1d4r", "2d4r", "1d6r") and family not in STENCILS:
        raise ValueError("unknown predictor family or stencil")
    return [f"{s}_xx{o}" for s in STENCILS if family == "all" or s.startswith(family) for o in range(3)]


def coefficients(predictor: str, six_grid: str = "legacy"):
    """The predictor's coefficient grid as [(c0, c1), ...]."""
    L = _bind(api.lib())
    n = C.c_uint64(0)
    if L.asz_sweep_coefs(predictor.encode(), six_grid.encode(), None, None, 0, C.byref(n)):
        raise ValueError(f"unknown predictor or grid: {predictor} {six_grid}")
    a, b = np.empty(n.value), np.empty(n.value)
    L.asz_sweep_coefs(predictor.encode(), six_grid.encode(), a.ctypes.data, b.ctypes.data, n.value, C.byref(n))
    return list(zip(a.tolist(), b.tolist()))


def targets(shape, predictor: str, mode: str = "legacy") -> np.ndarray:
    """(S, 3) coordinates of the targets in QB stream order, from the kernel's mapping run on the host."""
    L = _bind(api.lib())
    n = C.c_uint64(0)
    if L.asz_sweep_targets(api._dims(shape), predictor.encode(), mode.encode(), None, 0, C.byref(n)):
        raise ValueError(f"bad predictor or target mode: {predictor} {mode}")
    out = np.empty((n.value, 3), np.uint64)
    rc = L.asz_sweep_targets(api._dims(shape), predictor.encode(), mode.encode(), out.ctypes.data, n.value, C.byref(n))
    if rc:
        raise RuntimeError(f"target mapping inconsistent ({rc})")
    return out


def run(ctx: api.Context, data, predictor: str, rel_ebs, targets: str = "legacy", six_grid: str = "legacy"):
    """All rows of one predictor (rel_eb outer, coefficient inner). data: a float32 NumPy array or
    a contiguous float32 CUDA tensor. Returns (rows, (min_val, max_val))."""
    L = _bind(ctx._L)
    ebs = np.ascontiguousarray(rel_ebs, dtype=np.float64).reshape(-1)
    try:
        k = len(coefficients(predictor, six_grid))
    except ValueError:  # the library reports it with its message
        k = 0
    cap = max(1, len(ebs) * k)
    rows = (SweepRow * cap)()
    n = C.c_uint64(0)
    mm = (C.c_float * 2)()
    if api._is_cuda_tensor(data):
        import torch
        if data.dtype != torch.float32 or not data.is_contiguous():
            raise ValueError("device input must be a contiguous float32 tensor")
        ctx._use_torch_stream(data)
        try:
            rc = L.asz_sweep(ctx._c, C.c_void_p(data.data_ptr()), 1, api._dims(data.shape), predictor.encode(),
                             targets.encode(), six_grid.encode(), ebs.ctypes.data, len(ebs), rows, cap, C.byref(n), mm)
        finally:
            L.asz_set_stream(ctx._c, None)
    else:
        a = np.ascontiguousarray(data, dtype=np.float32)
        rc = L.asz_sweep(ctx._c, C.c_void_p(a.ctypes.data), 0, api._dims(a.shape), predictor.encode(), targets.encode(),
                         six_grid.encode(), ebs.ctypes.data, len(ebs), rows, cap, C.byref(n), mm)
    ctx._check(rc)
    return list(rows[: n.value]), (mm[0], mm[1])
