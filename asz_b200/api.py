"""Python binding of the C ABI in include/asz_b200.h (ctypes over the in-tree libasz_b200.so).

The functions mirror the reference's compressor/decompressor surface: ``compress`` takes a float32
field, an error bound, a predictor plan and the s1_compress tunables, and returns .asz bytes;
``decompress`` inverts it. Inputs may be NumPy arrays (host) or CUDA tensors (device pointers,
run on the caller's current stream). There is no CPU fallback: if the CUDA library is missing or
no GPU is present, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libasz_b200.so")
_LIB = None

ASZ_FAMILY_AUTO, ASZ_FAMILY_CUBIC, ASZ_FAMILY_QUINTIC = -1, 0, 1
ASZ_OK, ASZ_E_ARG, ASZ_E_DATA, ASZ_E_CUDA, ASZ_E_DEVICE, ASZ_E_UNSUPPORTED, ASZ_E_COMM = 0, -1, -2, -3, -4, -5, -6


class AszError(RuntimeError):
    """A call returned a nonzero status; the message is asz_last_error()."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("pivot_eb_ratio", C.c_float), ("eb_ratio", C.c_float), ("slope_ratio", C.c_float),
        ("block_pivot_ratio", C.c_uint64), ("max_layer_num", C.c_uint64),
        ("full_predictor_search_layer_num", C.c_uint64), ("generate_config_sample_stride", C.c_uint64),
        ("h1_block_sampling_num", C.c_uint64), ("stat_eb_ratio", C.c_float),
        ("predictor_family_suffix_layers", C.c_uint64), ("predictor_family_sample_blocks", C.c_uint64),
        ("predictor_family_sample_point_limit", C.c_uint64), ("predictor_family_sample_fraction_limit", C.c_float),
        ("predictor_family_coarse_probe_block_pivot_ratio", C.c_uint64),
        ("predictor_family_fine_probe_block_pivot_ratio", C.c_uint64),
        ("predictor_family_fine_eb_threshold", C.c_float), ("default_slope_invalid_ratio_threshold", C.c_float),
        ("default_slope_fallback", C.c_float), ("default_slope_eb_span", C.c_float),
        ("t_precision", C.c_int32), ("t_min", C.c_float), ("t_max", C.c_float), ("t_range_set", C.c_int32),
        ("predictor_family", C.c_int32), ("report_t_histogram", C.c_int32),
    ]


class Report(C.Structure):
    _fields_ = [
        ("data_range_s", C.c_double), ("default_slope_s", C.c_double), ("plan_s", C.c_double),
        ("family_s", C.c_double), ("core_s", C.c_double), ("huffman_s", C.c_double), ("zstd_s", C.c_double),
        ("h2d_s", C.c_double), ("d2h_s", C.c_double), ("total_s", C.c_double),
        ("min_val", C.c_float), ("max_val", C.c_float), ("abs_eb", C.c_float), ("default_slope", C.c_float),
        ("max_err", C.c_float), ("psnr", C.c_float), ("cr", C.c_float), ("br", C.c_float),
        ("t_fallback_count", C.c_uint64), ("pre_zstd_len", C.c_uint64), ("asz_len", C.c_uint64),
        ("layer_num", C.c_uint64), ("slope_max_invalid_ratio", C.c_float), ("slope_fallback_reason", C.c_int32),
        ("ambiguous_decisions", C.c_uint64), ("reruns", C.c_uint64), ("exact_groups", C.c_uint64),
        ("serial_groups", C.c_uint64), ("exact_window", C.c_uint64), ("exact_undecided", C.c_uint64),
        ("wide_groups", C.c_uint64), ("kernel_launches", C.c_uint64),
        ("plan_stats_s", C.c_double), ("plan_sample_s", C.c_double), ("plan_lossless_s", C.c_double),
        ("plan_search_layers", C.c_uint32), ("plan_best_dist", C.c_float * 64),
        ("family_selected", C.c_int32), ("family_fallback", C.c_int32),
        ("fam_suffix_layers", C.c_uint64), ("fam_blocks", C.c_uint64), ("fam_sampled_points", C.c_uint64),
        ("fam_budget", C.c_uint64), ("fam_probe_bpr", C.c_uint64), ("fam_points", C.c_uint64),
        ("fam_cubic_mse", C.c_longdouble), ("fam_quintic_mse", C.c_longdouble), ("fam_cubic_psnr", C.c_longdouble),
        ("fam_quintic_psnr", C.c_longdouble), ("fam_cubic_h1", C.c_longdouble), ("fam_quintic_h1", C.c_longdouble),
        ("fam_score_gain", C.c_longdouble),
        ("pivot_stride", C.c_uint32 * 3), ("block_shape", C.c_uint32 * 3), ("block_num", C.c_uint32 * 3),
        ("quintic", C.c_int32), ("plan", C.c_char * (64 * 11 + 1)),
    ]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            if isinstance(v, bytes):
                v = v.decode()
            elif hasattr(v, "__len__"):
                v = list(v)
            out[name] = v
        return out


class BatchReport(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("total_s", "h2d_s", "prep_s", "tune_s", "rounds_s", "encode_s", "zstd_s",
                                          "rounds_ms")] + \
               [(k, C.c_uint64) for k in ("input_bytes", "output_bytes", "kernel_launches")] + \
               [(k, C.c_uint32) for k in ("tuned_now", "graph_reused", "fields_fallback", "fast_ctas_per_sm",
                                          "round_ctas_per_sm", "tpl_shift")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def lib():
    """Load libasz_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built: run asz_b200.build.build() (make -C asz_b200/csrc)")
    L = C.CDLL(LIB_PATH)
    L.asz_default_params.argtypes = [C.POINTER(Params)]
    L.asz_create.argtypes = [C.c_int]
    L.asz_create.restype = C.c_void_p
    L.asz_destroy.argtypes = [C.c_void_p]
    L.asz_last_error.argtypes = [C.c_void_p]
    L.asz_last_error.restype = C.c_char_p
    L.asz_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.asz_compress.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.c_float, C.POINTER(Params),
                               C.c_char_p, C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_size_t), C.POINTER(Report)]
    L.asz_compress_with_t.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.c_float,
                                      C.POINTER(Params), C.c_char_p, C.c_void_p, C.c_uint64,
                                      C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_size_t), C.POINTER(Report)]
    L.asz_compress_batch.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.c_float,
                                     C.POINTER(Params), C.c_char_p, C.c_void_p, C.POINTER(C.c_size_t),
                                     C.POINTER(Report), C.POINTER(BatchReport)]
    L.asz_compress_batch_with_t.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_int, C.POINTER(C.c_uint64),
                                            C.c_float, C.POINTER(Params), C.c_char_p, C.c_void_p, C.POINTER(C.c_uint64),
                                            C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(Report), C.POINTER(BatchReport)]
    L.asz_decompress.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_uint64), C.c_float,
                                 C.POINTER(Params), C.c_void_p, C.c_int, C.POINTER(Report)]
    L.asz_free.argtypes = [C.c_void_p]
    L.asz_compress_stats.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    for name, elem in (("asz_debug_qb", None), ("asz_debug_t", None), ("asz_debug_recon", None),
                       ("asz_debug_pre_zstd", None)):
        f = getattr(L, name)
        f.restype = C.c_uint64
    L.asz_debug_qb.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
    L.asz_debug_t.argtypes = [C.c_void_p, C.c_void_p]
    L.asz_debug_recon.argtypes = [C.c_void_p, C.c_void_p]
    L.asz_debug_pre_zstd.argtypes = [C.c_void_p, C.c_void_p]
    L.asz_debug_proxies.argtypes = [C.c_void_p, C.c_void_p]
    L.asz_set_tsel_mode.argtypes = [C.c_void_p, C.c_int]
    L.asz_debug_proxies.restype = C.c_uint64
    L.asz_error_stats_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_double, C.c_void_p,
                                          C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_char_p, C.c_size_t]
    L.asz_slab_planes.argtypes = [C.POINTER(C.c_uint64), C.c_void_p, C.c_char_p, C.c_uint64, C.c_uint64,
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.asz_compress_slab.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.c_uint64,
                                    C.c_uint64, C.c_float, C.POINTER(Params), C.c_char_p,
                                    C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_size_t), C.POINTER(Report)]
    _LIB = L
    return L


def default_params(**kw) -> Params:
    p = Params()
    lib().asz_default_params(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def _family_code(family):
    if family is None or family == "auto":
        return ASZ_FAMILY_AUTO
    return {"cubic": ASZ_FAMILY_CUBIC, "quintic": ASZ_FAMILY_QUINTIC}[family]


def _dims(shape):
    if len(shape) != 3:
        raise ValueError("fields are three-dimensional")
    return (C.c_uint64 * 3)(*[int(s) for s in shape])


def _is_cuda_tensor(x):
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _check_device_field(x, device: int, what: str, numel: int | None = None):
    """Refuse a CUDA tensor the library would misread: it must be float32, contiguous, on the
    context's device and, when numel is given, hold exactly that many values. The library reads
    and writes such buffers through raw pointers, so a mismatch would run past the tensor."""
    import torch
    if x.dtype != torch.float32:
        raise ValueError(f"{what} must be a float32 tensor, not {x.dtype}")
    if not x.is_contiguous():
        raise ValueError(f"{what} must be contiguous")
    if x.device.index != device:
        raise ValueError(f"{what} is on {x.device}, the context uses cuda:{device}")
    if numel is not None and x.numel() != numel:
        raise ValueError(f"{what} holds {x.numel()} values, the shape needs {numel}")


def error_stats_noalloc(x, y, value_range: float):
    """max |x - y| and PSNR of two equal-size float32 CUDA tensors, computed without allocating
    (fixed library scratch). Runs on torch's current stream of x's device; returns (max_err, psnr)."""
    import torch
    if not (_is_cuda_tensor(x) and _is_cuda_tensor(y)) or x.dtype != torch.float32 or y.dtype != torch.float32:
        raise ValueError("x and y must be float32 CUDA tensors")
    if x.numel() != y.numel() or not x.is_contiguous() or not y.is_contiguous():
        raise ValueError("x and y must be contiguous and of equal size")
    m, ps = C.c_double(), C.c_double()
    err = C.create_string_buffer(256)
    with torch.cuda.device(x.device):
        rc = lib().asz_error_stats_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), x.numel(),
                                           float(value_range),
                                           C.c_void_p(torch.cuda.current_stream(x.device).cuda_stream),
                                           C.byref(m), C.byref(ps), err, 256)
    if rc != ASZ_OK:
        raise AszError(rc, err.value.decode(errors="replace"))
    return m.value, ps.value


class Context:
    """One CUDA context: a stream and the device buffers reused across calls."""

    def __init__(self, device: int = 0):
        self._L = lib()
        self._c = self._L.asz_create(int(device))
        if not self._c:
            raise RuntimeError(f"asz_create({device}) failed: no usable CUDA device")
        self.device = device

    def close(self):
        if self._c:
            self._L.asz_destroy(self._c)
            self._c = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise AszError(rc, self._L.asz_last_error(self._c).decode())

    def _use_torch_stream(self, x):
        import torch
        self._L.asz_set_stream(self._c, C.c_void_p(torch.cuda.current_stream(x.device).cuda_stream))

    def compress(self, data, rel_eb: float, plan: str | None, family="cubic", params: Params | None = None):
        """Compress a float32 field; returns (asz bytes, Report)."""
        p = params if params is not None else default_params()
        p.predictor_family = _family_code(family) if family is not None else p.predictor_family
        out = C.POINTER(C.c_uint8)()
        n = C.c_size_t(0)
        rep = Report()
        if _is_cuda_tensor(data):
            _check_device_field(data, self.device, "device input")
            self._use_torch_stream(data)
            rc = self._L.asz_compress(self._c, C.c_void_p(data.data_ptr()), 1, _dims(data.shape), C.c_float(rel_eb),
                                      C.byref(p), plan.encode() if plan else None, C.byref(out), C.byref(n), C.byref(rep))
            self._L.asz_set_stream(self._c, None)
        else:
            a = np.ascontiguousarray(data, dtype=np.float32)
            rc = self._L.asz_compress(self._c, C.c_void_p(a.ctypes.data), 0, _dims(a.shape), C.c_float(rel_eb),
                                      C.byref(p), plan.encode() if plan else None, C.byref(out), C.byref(n), C.byref(rep))
        self._check(rc)
        try:
            blob = C.string_at(out, n.value)
        finally:
            self._L.asz_free(out)
        return blob, rep

    def decompress(self, blob: bytes, shape, rel_eb: float, params: Params | None = None, out=None):
        """Decompress .asz bytes; returns a NumPy array, or fills the CUDA tensor `out`."""
        p = params if params is not None else default_params()
        rep = Report()
        numel = 1
        for s_ in shape:
            numel *= int(s_)
        if out is not None:
            if not _is_cuda_tensor(out):
                raise ValueError("out must be a CUDA tensor (omit it to get a NumPy array)")
            _check_device_field(out, self.device, "out", numel)
        buf = C.create_string_buffer(bytes(blob), len(blob))
        if out is not None:
            self._use_torch_stream(out)
            rc = self._L.asz_decompress(self._c, buf, len(blob), _dims(shape), C.c_float(rel_eb), C.byref(p),
                                        C.c_void_p(out.data_ptr()), 1, C.byref(rep))
            self._L.asz_set_stream(self._c, None)
            self._check(rc)
            return out, rep
        res = np.empty(tuple(int(s) for s in shape), dtype=np.float32)
        rc = self._L.asz_decompress(self._c, buf, len(blob), _dims(shape), C.c_float(rel_eb), C.byref(p),
                                    C.c_void_p(res.ctypes.data), 0, C.byref(rep))
        self._check(rc)
        return res, rep

    def compress_with_t(self, data, rel_eb: float, plan: str, family: str, params: Params | None, t_int):
        """Compress with given block-major t codes (NumPy or torch int64, blocks x layers) instead of
        the coefficient selection; returns (asz bytes, Report)."""
        p = params if params is not None else default_params()
        p.predictor_family = _family_code(family)
        if hasattr(t_int, "detach"):
            t_int = t_int.detach().cpu().numpy()
        codes = np.ascontiguousarray(t_int, dtype=np.int64)
        out = C.POINTER(C.c_uint8)()
        n = C.c_size_t(0)
        rep = Report()
        if _is_cuda_tensor(data):
            _check_device_field(data, self.device, "device input")
            self._use_torch_stream(data)
            rc = self._L.asz_compress_with_t(self._c, C.c_void_p(data.data_ptr()), 1, _dims(data.shape), C.c_float(rel_eb),
                                             C.byref(p), plan.encode(), C.c_void_p(codes.ctypes.data), codes.size,
                                             C.byref(out), C.byref(n), C.byref(rep))
            self._L.asz_set_stream(self._c, None)
        else:
            a = np.ascontiguousarray(data, dtype=np.float32)
            rc = self._L.asz_compress_with_t(self._c, C.c_void_p(a.ctypes.data), 0, _dims(a.shape), C.c_float(rel_eb),
                                             C.byref(p), plan.encode(), C.c_void_p(codes.ctypes.data), codes.size,
                                             C.byref(out), C.byref(n), C.byref(rep))
        self._check(rc)
        try:
            blob = C.string_at(out, n.value)
        finally:
            self._L.asz_free(out)
        return blob, rep

    def compress_batch(self, fields, rel_eb: float, plan: str, family: str = "cubic", params: Params | None = None,
                       t_tables=None):
        """Compress several fields (all NumPy arrays, or all contiguous float32 CUDA tensors on one
        stream) with one plan; returns (list of asz bytes, list of Report, BatchReport). t_tables:
        optional per-field block-major t codes (NumPy or torch int64) replacing the selection."""
        p = params if params is not None else default_params()
        p.predictor_family = _family_code(family)
        n = len(fields)
        ptrs = (C.c_void_p * n)()
        dims = (C.c_uint64 * (3 * n))()
        keep = []
        on_dev = _is_cuda_tensor(fields[0])
        for i, x in enumerate(fields):
            if on_dev:
                if not _is_cuda_tensor(x):
                    raise ValueError("fields must be all CUDA tensors or all host arrays")
                _check_device_field(x, self.device, f"device input {i}")
                if x.device != fields[0].device:
                    raise ValueError("device inputs must share one device")
                ptrs[i] = x.data_ptr()
            else:
                a = np.ascontiguousarray(x, dtype=np.float32)
                keep.append(a)
                ptrs[i] = a.ctypes.data
            for k in range(3):
                dims[3 * i + k] = int(x.shape[k])
        outs = (C.POINTER(C.c_uint8) * n)()
        lens = (C.c_size_t * n)()
        reps = (Report * n)()
        br = BatchReport()
        if on_dev:
            self._use_torch_stream(fields[0])
        try:
            if t_tables is None:
                rc = self._L.asz_compress_batch(self._c, n, ptrs, 1 if on_dev else 0, dims, C.c_float(rel_eb), C.byref(p),
                                                plan.encode(), outs, lens, reps, C.byref(br))
            else:
                tabs = [np.ascontiguousarray(t.detach().cpu().numpy() if hasattr(t, "detach") else t, dtype=np.int64)
                        for t in t_tables]
                keep.extend(tabs)
                tptr = (C.c_void_p * n)(*[t.ctypes.data for t in tabs])
                tlen = (C.c_uint64 * n)(*[t.size for t in tabs])
                rc = self._L.asz_compress_batch_with_t(self._c, n, ptrs, 1 if on_dev else 0, dims, C.c_float(rel_eb),
                                                       C.byref(p), plan.encode(), tptr, tlen, outs, lens, reps,
                                                       C.byref(br))
        finally:
            if on_dev:
                self._L.asz_set_stream(self._c, None)
        self._check(rc)
        blobs = []
        for i in range(n):
            blobs.append(C.string_at(outs[i], lens[i]))
            self._L.asz_free(outs[i])
        return blobs, list(reps), br

    def set_tsel_mode(self, mode: int):
        """0: certified fast path + exact replay for the rest, one launch per round (default);
        1: exact replay everywhere; 2: as 0 with the rounds of all-axis-2 plans fused."""
        self._check(self._L.asz_set_tsel_mode(self._c, int(mode)))

    def stats(self):
        m, ps = C.c_double(), C.c_double()
        self._check(self._L.asz_compress_stats(self._c, C.byref(m), C.byref(ps)))
        return m.value, ps.value

    # Internals of the last compress call (parity checks).
    def debug_qb(self, stream: int) -> np.ndarray:
        n = self._L.asz_debug_qb(self._c, stream, None)
        a = np.empty(n, np.int32)
        if n:
            self._L.asz_debug_qb(self._c, stream, C.c_void_p(a.ctypes.data))
        return a

    def debug_t(self) -> np.ndarray:
        n = self._L.asz_debug_t(self._c, None)
        a = np.empty(n, np.int64)
        if n:
            self._L.asz_debug_t(self._c, C.c_void_p(a.ctypes.data))
        return a

    def debug_recon(self) -> np.ndarray:
        n = self._L.asz_debug_recon(self._c, None)
        a = np.empty(n, np.float32)
        if n:
            self._L.asz_debug_recon(self._c, C.c_void_p(a.ctypes.data))
        return a

    def debug_proxies(self) -> np.ndarray:
        """(rounds, blocks, 10) float32: h1 for the five t candidates, then the log10f arguments."""
        n = self._L.asz_debug_proxies(self._c, None)
        a = np.empty(n, np.float32)
        if n:
            self._L.asz_debug_proxies(self._c, C.c_void_p(a.ctypes.data))
        return a

    def debug_pre_zstd(self) -> bytes:
        n = self._L.asz_debug_pre_zstd(self._c, None)
        a = (C.c_uint8 * max(n, 1))()
        if n:
            self._L.asz_debug_pre_zstd(self._c, a)
        return bytes(a)[:n]
