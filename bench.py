"""Benchmark: ASZ compression hot path on B200 (one JSON line on rank 0).

Workload: one 512^3 float32 field (k^-5/3 Gaussian random field plus a tanh front of width 4
voxels on a random plane, amplitude 10x the field's std, seeded), REL 1e-3, the fixed plan
"cubic2_012" on every level (9 rounds), cubic family, block_pivot_ratio 3 (the reference launcher's
setting for REL > 1e-4).

  value  compress throughput in input GB/s with the field resident in HBM. Each step is one full
         compression to the pre-zstd stream (range, default slope, all rounds with per-block t,
         histograms, Huffman codes and encoding). The final libzstd stage is timed separately.
  e2e    the same through the C ABI from pinned host memory to .asz bytes on the host, with the
         host->device copy, the device->host copy of the stream and libzstd inside the timed region.
Decompression throughput is reported beside them. The field (512 MiB) is larger than L2 (126 MB),
so no flush is needed between steps.

Multi-GPU: fields are independent, so each rank compresses its own field (weak scaling, no
collective on the data path); value = total input bytes / max-over-ranks time.

--impl reference times the reference's own CPU compressor (oracle/_ref/s1_compress, built from
the reference sources) on a bounded slab of the same field.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPE = (512, 512, 512)
C1_SHAPE = (100, 500, 500)
REL_EB = 1e-3
PLAN = ",".join(["cubic2_012"] * 9)
FAMILY = "cubic"
BPR = 3
METRIC = "compress/decompress GB/s at REL 1e-3 (bit-exact); tune time & CR vs plain at same eb"
WORKLOAD = "512^3 float32 k^-5/3 GRF + tanh front, REL 1e-3, plan cubic2_012 x9, cubic, block_pivot_ratio 3"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def cpu_baseline(field_np, workdir):
    """The reference s1_compress (one process, one thread) on the full field, same plan, error
    bound and flags: about 20 s of host work for 512^3."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    exe = O.ref_binary("s1_compress")
    if exe is None:
        return None
    inp = os.path.join(workdir, "field.f32")
    out = os.path.join(workdir, "field.asz")
    np.ascontiguousarray(field_np).tofile(inp)
    argv = [exe, "-f", "-i", inp, "-3", *[str(s) for s in field_np.shape], "-M", "REL", f"{REL_EB:.17g}",
            "--block-pivot-ratio", str(BPR), "--predictor-family", FAMILY, "-z", out, "--predictor-plan", PLAN]
    t0 = time.perf_counter()
    r = subprocess.run(argv, capture_output=True, text=True)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        return None
    comp = None
    for line in r.stdout.splitlines():
        if line.startswith("Compression time:"):
            comp = float(line.split(":")[1].split()[0])
    shape = "x".join(map(str, field_np.shape))
    return {"value": field_np.nbytes / 1e9 / wall, "unit": "GB/s", "cores": 1, "kind": "reference",
            "sample": f"reference s1_compress on the full {shape} field of this run, one process, wall time"
                      + (f" (its own 'Compression time' {comp:.3f} s)" if comp else "")}


def bench_config(shape, world):
    """The `config` object of both arms' JSON lines (identical, so the two lines compare)."""
    n = shape[0] * shape[1] * shape[2]
    workload = WORKLOAD if tuple(shape) == SHAPE else WORKLOAD.replace("512^3", "x".join(map(str, shape)))
    return {"workload": workload, "field": "asz_b200.fields.c2_field(seed=2 + rank), generated on the host",
            "inputs": f"{4 * n / 2**20:.0f} MiB per field; "
                      + ("> L2, no flush needed" if 4 * n > 126e6 else "fits L2 (profiling size only)"),
            "parallelism": f"replicas x{world}"}


def make_bench_field(rank, shape):
    """The benchmark field of `rank`: the C2 recipe from seed 2 + rank (NumPy, on the host). Rank 0's
    512^3 field is the one tests/golden/fullsize.json records the reference's output for."""
    from asz_b200 import fields
    return fields.c2_field(seed=2 + rank, shape=tuple(shape))


def reference_parity(x_host, blob, y, rank):
    """This run's .asz and decompressed output against the reference's, recorded for the same input
    bytes by tests/golden/make_fullsize.py (case c2_cubic_0.001: this workload). None when the field
    is not the recorded one (other ranks, other shapes)."""
    import hashlib
    try:
        with open(os.path.join(ROOT, "tests", "golden", "fullsize.json")) as f:
            fix = json.load(f)
    except OSError:
        return None
    if rank != 0 or hashlib.sha256(x_host.tobytes()).hexdigest() != fix["fields"]["c2"]["sha256"]:
        return None
    case = next(c for c in fix["cases"] if c["name"] == "c2_cubic_0.001")
    dec = y.cpu().numpy().tobytes()
    return {"case": case["name"], "asz_equal": hashlib.sha256(blob).hexdigest() == case["asz_sha256"],
            "decompressed_equal": hashlib.sha256(dec).hexdigest() == case["decompressed_sha256"],
            "source": "SHA-256 digests of the reference binaries' output on the same input (tests/golden/fullsize.json)"}


def _usable_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def _available_bytes():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 16 << 30


def _run_pool(argvs, workers):
    """Run the command lines with at most `workers` at a time; returns the wall time."""
    import concurrent.futures as cf
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(workers) as ex:
        for r in ex.map(lambda a: subprocess.run(a, capture_output=True, text=True), argvs):
            if r.returncode != 0:
                raise RuntimeError(f"reference run failed: {r.stderr.strip()[:200]}")
    return time.perf_counter() - t0


def run_reference_arm(args):
    """The reference's own compressor (oracle/_ref/s1_compress, compiled from the reference sources
    with its flags) on the same field, error bound, plan and flags as this build's arm. One step is
    one full compression of the 512^3 field. The reference is single-threaded, so the steps run as
    concurrent processes, as many as the host's cores and memory allow: value is the aggregate
    input GB/s of the timed steps over their wall time. Its decompressor is timed the same way."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    exe, dexe = O.ref_binary("s1_compress"), O.ref_binary("s1_decompress")
    if exe is None or dexe is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference binaries not built (make -C oracle ref)"}))
        return
    shape = tuple(int(v) for v in args.shape.split(","))
    field = make_bench_field(0, shape)
    nbytes = field.nbytes
    # About 2.2 GB of host memory per 512^3 compression (input, its working copy, QB streams).
    per_proc = 4.5 * nbytes + (64 << 20)
    workers = max(1, min(args.steps, _usable_cores(), int(_available_bytes() * 0.8 // per_proc)))
    with tempfile.TemporaryDirectory() as wd:
        inp = os.path.join(wd, "field.f32")
        field.tofile(inp)
        del field
        common = ["-f", "-i", inp, "-3", *map(str, shape), "-M", "REL", f"{REL_EB:.17g}",
                  "--block-pivot-ratio", str(BPR), "--predictor-family", FAMILY]

        def comp(k):
            return [exe, *common, "-z", os.path.join(wd, f"o{k}.asz"), "--predictor-plan", PLAN]

        def decomp(k):
            return [dexe, *common, "-z", os.path.join(wd, f"o{k % workers}.asz"), "-o", os.path.join(wd, f"r{k % workers}.f32")]

        _run_pool([comp(k) for k in range(args.warmup)], workers)
        dt = _run_pool([comp(k) for k in range(args.steps)], workers)
        asz_len = os.path.getsize(os.path.join(wd, "o0.asz"))
        ddt = _run_pool([decomp(k) for k in range(args.steps)], workers)
    gbs = nbytes * args.steps / 1e9 / dt
    dgbs = nbytes * args.steps / 1e9 / ddt
    sample = (f"reference s1_compress on the full {'x'.join(map(str, shape))} field per step, {workers} single-threaded "
              f"processes at a time ({_usable_cores()} usable cores), aggregate input GB/s")
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": gbs, "unit": "GB/s", "n_gpus": args.gpus,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1000 / args.steps,
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                      "data": "synthetic", "config": bench_config(shape, 1),
                      "decompress": {"value": dgbs, "unit": "GB/s", "ms_per_step": ddt * 1000 / args.steps},
                      "cr": nbytes / asz_len, "concurrent_processes": workers,
                      "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": workers, "kind": "reference", "sample": sample},
                      "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shape", default="512,512,512", help="field shape (smaller shapes are for profiler captures)")
    ap.add_argument("--no-tune", action="store_true", help="skip the plan-search / family-selection measurement")
    ap.add_argument("--no-batch", action="store_true", help="skip the 48-field batch measurement")
    ap.add_argument("--no-series", action="store_true", help="skip the 16-step time-series measurement")
    ap.add_argument("--no-sweep", action="store_true", help="skip the prediction-sweep (s2_many_prediction) measurement")
    args = ap.parse_args()
    shape = tuple(int(v) for v in args.shape.split(","))
    if args.impl == "reference":
        run_reference_arm(args)
        return
    import ctypes as C

    import torch

    import asz_b200.api as api
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    x_host = make_bench_field(rank, shape)
    x = torch.from_numpy(x_host).to(dev)
    N = x.numel()
    p = api.default_params(block_pivot_ratio=BPR)
    ctx = api.Context(local)
    L = api.lib()
    L.asz_profile_enable.argtypes = [C.c_void_p, C.c_int]
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize(dev)

    y = torch.empty_like(x)
    # The timed loops call the C ABI directly (the reference-facing boundary), on torch's stream.
    L.asz_set_stream(ctx._c, C.c_void_p(stream.cuda_stream))
    p.predictor_family = api.ASZ_FAMILY_CUBIC
    dims = api._dims(shape)
    plan_b = PLAN.encode()
    outp = C.POINTER(C.c_uint8)()
    outn = C.c_size_t(0)
    rep = api.Report()

    def compress_abi(ptr, on_device):
        rc = L.asz_compress(ctx._c, C.c_void_p(ptr), on_device, dims, C.c_float(REL_EB), C.byref(p), plan_b,
                            C.byref(outp), C.byref(outn), C.byref(rep))
        if rc:
            raise api.AszError(rc, L.asz_last_error(ctx._c).decode())
        L.asz_free(outp)
        return rep

    blob = None
    for _ in range(args.warmup):
        blob, _r = ctx.compress(x, REL_EB, PLAN, FAMILY, p)
        L.asz_set_stream(ctx._c, C.c_void_p(stream.cuda_stream))
        ctx.decompress(blob, shape, REL_EB, p, out=y)
        L.asz_set_stream(ctx._c, C.c_void_p(stream.cuda_stream))
    blob_np = np.frombuffer(blob, dtype=np.uint8)
    blob_ptr = C.c_void_p(blob_np.ctypes.data)
    drep = api.Report()

    def decompress_abi(out_ptr, on_device):
        rc = L.asz_decompress(ctx._c, blob_ptr, len(blob), dims, C.c_float(REL_EB), C.byref(p), C.c_void_p(out_ptr),
                              on_device, C.byref(drep))
        if rc:
            raise api.AszError(rc, L.asz_last_error(ctx._c).decode())
        return drep

    # Compress, device-resident input. libzstd and the device->host copy of the stream run inside
    # each call; their measured durations are taken out of `value` and reported apart.
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    zstd_s = d2h_s = 0.0
    launches = 0
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            r = compress_abi(x.data_ptr(), 1)
            zstd_s += r.zstd_s
            d2h_s += r.d2h_s
            launches += r.kernel_launches
        ev1.record(stream)
        barrier()
    call_ms = ev0.elapsed_time(ev1)
    core_ms = call_ms - (zstd_s + d2h_s) * 1000
    pre_zstd_len = int(rep.pre_zstd_len)
    asz_len = int(rep.asz_len)
    # Decompress into device memory (zstd and the stream's host->device copy taken out likewise).
    barrier()
    dz_s = dh2d_s = 0.0
    ev0.record(stream)
    for _ in range(args.steps):
        r = decompress_abi(y.data_ptr(), 1)
        dz_s += r.zstd_s
        dh2d_s += r.h2d_s
    ev1.record(stream)
    barrier()
    dec_call_ms = ev0.elapsed_time(ev1)
    dec_ms = dec_call_ms - (dz_s + dh2d_s) * 1000
    # Parity spot check of this run: decompression equals the compressor's reconstruction.
    blob, rep1 = ctx.compress(x, REL_EB, PLAN, FAMILY, p)
    rec = torch.from_numpy(ctx.debug_recon()).to(dev).view(shape)
    ctx.decompress(blob, shape, REL_EB, p, out=y)
    torch.cuda.synchronize(dev)
    bit_exact = bool(torch.equal(rec.view(torch.int32), y.view(torch.int32)))
    max_err = float((y - x).abs().max().item())
    del rec
    parity = reference_parity(x_host, blob, y, rank)
    # Profile of one compression and one decompression (per kernel family, CUDA events).
    L.asz_set_stream(ctx._c, C.c_void_p(stream.cuda_stream))
    L.asz_profile_enable(ctx._c, 1)
    compress_abi(x.data_ptr(), 1)
    entries = (PROFILE_ENTRY * 64)()
    n = L.asz_profile_read(ctx._c, entries, 64, 1)
    prof = {entries[i].name.decode(): {"launches": entries[i].launches, "ms": entries[i].ms, "bytes": entries[i].bytes}
            for i in range(min(n, 64))}
    decompress_abi(y.data_ptr(), 1)
    n = L.asz_profile_read(ctx._c, entries, 64, 1)
    L.asz_profile_enable(ctx._c, 0)
    prof_dec = {entries[i].name.decode(): {"launches": entries[i].launches, "ms": entries[i].ms, "bytes": entries[i].bytes}
                for i in range(min(n, 64))}
    # Host wall-time phases ("host:*") are reported apart from the device kernel families.
    host_phases = {k[5:]: round(v["ms"], 3) for k, v in prof.items() if k.startswith("host:")}
    host_phases_dec = {k[5:]: round(v["ms"], 3) for k, v in prof_dec.items() if k.startswith("host:")}
    prof = {k: v for k, v in prof.items() if not k.startswith("host:")}
    prof_dec = {k: v for k, v in prof_dec.items() if not k.startswith("host:")}
    # End to end from pinned host memory to .asz bytes on the host (everything included), and back.
    xh = x.cpu().pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        r = compress_abi(xh.data_ptr(), 0)
    ev1.record(stream)
    barrier()
    e2e_ms = ev0.elapsed_time(ev1)
    ev0.record(stream)
    for _ in range(args.steps):
        decompress_abi(yh.data_ptr(), 0)
    ev1.record(stream)
    barrier()
    e2e_dec_ms = ev0.elapsed_time(ev1)
    # The same steps, several calls in flight: a host thread per context (its own stream and
    # buffers), so one call's libzstd and copies overlap another's kernels. Host wall clock around
    # all steps, device idle on both sides.
    workers = E2E_WORKERS if world == 1 else E2E_WORKERS_PER_RANK
    e2e_pipe_ms, e2e_pipe_dec_ms = e2e_pipelined(api, L, local, dims, p, plan_b, xh, yh, blob, args.steps, barrier, workers)
    # Tuning (config 0's form): a C1-shaped field with the plan search and the family selector,
    # beside a fixed cyclic plan at the same error bound. Device-resident input.
    tune = None
    if not args.no_tune:
        from asz_b200 import fields
        c1 = torch.from_numpy(fields.c1_field(seed=7 + rank, shape=C1_SHAPE)).to(dev)
        c1dims = api._dims(C1_SHAPE)
        pa = api.default_params(block_pivot_ratio=BPR)  # family left automatic
        pc = api.default_params(block_pivot_ratio=BPR)
        pc.predictor_family = api.ASZ_FAMILY_CUBIC
        tr = api.Report()

        def run(params, plan):
            rc = L.asz_compress(ctx._c, C.c_void_p(c1.data_ptr()), 1, c1dims, C.c_float(REL_EB), C.byref(params), plan,
                                C.byref(outp), C.byref(outn), C.byref(tr))
            if rc:
                raise api.AszError(rc, L.asz_last_error(ctx._c).decode())
            L.asz_free(outp)
            return tr

        run(pa, None)  # warm-up
        barrier()
        t0 = time.perf_counter()
        r = run(pa, None)
        auto_s = time.perf_counter() - t0
        _, auto_psnr = ctx.stats()
        auto = {"plan_search_ms": r.plan_s * 1e3,
                "plan_search_phases_ms": {"statistics": r.plan_stats_s * 1e3, "sample_prediction": r.plan_sample_s * 1e3,
                                          "lossless_estimation": r.plan_lossless_s * 1e3},
                "family_selection_ms": r.family_s * 1e3, "call_ms": auto_s * 1e3,
                "zstd_ms": r.zstd_s * 1e3, "cr": float(r.cr), "psnr_db": auto_psnr, "family": "quintic" if r.quintic else "cubic",
                "layers": int(r.layer_num), "plan": r.plan.decode()}
        cyc = ",".join(["cubic0_012", "cubic1_012", "cubic2_012"] * 4)
        run(pc, cyc.encode())
        t0 = time.perf_counter()
        r = run(pc, cyc.encode())
        fixed_s = time.perf_counter() - t0
        _, fixed_psnr = ctx.stats()
        fixed = {"call_ms": fixed_s * 1e3, "zstd_ms": r.zstd_s * 1e3, "cr": float(r.cr), "psnr_db": fixed_psnr, "plan": cyc}
        tune = {"field": "x".join(map(str, C1_SHAPE)) + " k^-11/3 GRF + 20 blobs + 1e-4 noise, REL 1e-3, block_pivot_ratio 3",
                "auto": auto, "fixed_cyclic": fixed, "timing": "host wall clock around one C-ABI call each"}
        del c1
    grad_tune = None if args.no_tune else grad_tune_section(ctx, L, dev, rank, barrier)
    sweep = None if args.no_sweep else sweep_section(ctx, dev, rank, with_reference=not args.no_cpu_baseline)
    batch = None if args.no_batch else batch_section(ctx, dev, rank)
    series = None if args.no_series else series_section(ctx, dev, rank)
    L.asz_set_stream(ctx._c, None)
    # Max over ranks.
    times = torch.tensor([core_ms, dec_ms, e2e_ms, e2e_dec_ms, e2e_pipe_ms, e2e_pipe_dec_ms], device=dev)
    if pg:
        pg.all_reduce(times, op=pg.ReduceOp.MAX)
    core_ms, dec_ms, e2e_ms, e2e_dec_ms, e2e_pipe_ms, e2e_pipe_dec_ms = times.tolist()
    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return
    total_bytes = 4.0 * N * world
    comp_gbs = total_bytes * args.steps / (core_ms / 1000) / 1e9
    dec_gbs = total_bytes * args.steps / (dec_ms / 1000) / 1e9
    e2e_gbs = total_bytes * args.steps / (e2e_pipe_ms / 1000) / 1e9
    e2e_dec_gbs = total_bytes * args.steps / (e2e_pipe_dec_ms / 1000) / 1e9
    e2e_one_gbs = total_bytes * args.steps / (e2e_ms / 1000) / 1e9
    e2e_one_dec_gbs = total_bytes * args.steps / (e2e_dec_ms / 1000) / 1e9
    peak, peak_kind = measured_peaks()
    # Dominant kernel family: algorithmic bytes of its launches over their CUDA-event time.
    roofline = None
    ranked = sorted(((k, v) for k, v in prof.items() if v["bytes"]), key=lambda kv: -kv[1]["ms"])
    if ranked:
        name, t = ranked[0]
        ach = t["bytes"] / (t["ms"] / 1000) / 1e9
        roofline = {"bound": "hbm", "kernel": name, "launches": t["launches"], "achieved": ach, "peak": peak,
                    "unit": "GB/s", "frac": ach / peak, "peak_source": peak_kind,
                    "traffic": TRAFFIC_PER_LAUNCH.get(name)}
    # Whole path: 4N read + the stream written, over the compress device time.
    path_ach = (4.0 * N + pre_zstd_len) / (core_ms / args.steps / 1000) / 1e9
    roofline_path = {"bound": "hbm", "achieved": path_ach, "peak": peak, "unit": "GB/s", "frac": path_ach / peak,
                     "bytes_per_step": 4 * N + pre_zstd_len}
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        with tempfile.TemporaryDirectory() as wd:
            cpu = cpu_baseline(x_host, wd)
    out = {
        "metric": METRIC, "value": comp_gbs, "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": core_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": bench_config(shape, world),
        "value_excludes": "libzstd and host<->device copies (timed inside the call, reported apart)",
        "decompress": {"value": dec_gbs, "unit": "GB/s", "ms_per_step": dec_ms / args.steps},
        "zstd_ms_per_step": zstd_s * 1000 / args.steps, "d2h_ms_per_step": d2h_s * 1000 / args.steps,
        "zstd_decompress_ms_per_step": dz_s * 1000 / args.steps,
        "e2e": {"value": e2e_gbs, "unit": "GB/s", "h2d_bytes_per_step": 4 * N, "d2h_bytes_per_step": pre_zstd_len,
                "ms_per_step": e2e_pipe_ms / args.steps, "calls_in_flight": workers,
                "includes": "every step one C-ABI call from pinned host memory to .asz bytes on the host: H2D, all GPU "
                            "stages, D2H of the stream, libzstd level 3",
                "timing": f"host wall clock around all steps, {workers} host threads each with its own context "
                          "taking steps in turn (one call's libzstd overlaps the others' copies and kernels)",
                "one_call_at_a_time": {"value": e2e_one_gbs, "ms_per_step": e2e_ms / args.steps}},
        "e2e_decompress": {"value": e2e_dec_gbs, "unit": "GB/s", "h2d_bytes_per_step": pre_zstd_len,
                           "d2h_bytes_per_step": 4 * N, "ms_per_step": e2e_pipe_dec_ms / args.steps,
                           "calls_in_flight": workers,
                           "one_call_at_a_time": {"value": e2e_one_dec_gbs, "ms_per_step": e2e_dec_ms / args.steps}},
        "cr": float(4 * N / asz_len), "pre_zstd_bytes": pre_zstd_len, "bit_exact_roundtrip": bit_exact,
        "parity_vs_reference": parity,
        "max_err_over_eb": max_err / rep1.abs_eb,
        "t_fallback_count": int(rep1.t_fallback_count), "ambiguous_decisions": int(rep1.ambiguous_decisions),
        "reruns": int(rep1.reruns),
        "exact_groups": int(rep1.exact_groups), "serial_groups": int(rep1.serial_groups),
        "exact_window": int(rep1.exact_window), "exact_undecided": int(rep1.exact_undecided),
        "wide_groups": int(rep1.wide_groups),
        "roofline": roofline, "roofline_path": roofline_path, "profile": prof, "host_phases_ms": host_phases,
        "decompress_profile": prof_dec, "decompress_host_phases_ms": host_phases_dec,
        "cpu_baseline": cpu, "clocks": clocks.summary(),
        "gpu_launches": int(launches), "tune": tune, "grad_tune": grad_tune, "batch": batch, "series": series,
        "sweep": sweep,
    }
    print(json.dumps(out))
    if pg:
        pg.destroy_process_group()


import ctypes as _C  # noqa: E402

C4_SHAPE = (256, 256, 256)


def grf_torch(seed, shape, alpha, device):
    """Unit-variance Gaussian random field with P(k) ~ k^-alpha, generated on the device."""
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    spec = torch.fft.rfftn(torch.randn(shape, generator=g, device=device, dtype=torch.float32))
    k = [torch.fft.fftfreq(n, device=device) * n for n in shape[:-1]] + [torch.fft.rfftfreq(shape[-1], device=device) * shape[-1]]
    kk = (k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2).sqrt_()
    kk[0, 0, 0] = 1.0
    amp = kk.pow_(-alpha / 2.0)
    amp[0, 0, 0] = 0.0
    f = torch.fft.irfftn(spec * amp, s=shape)
    f -= f.mean()
    f /= f.std()
    return f.contiguous()


C5_SHAPE = (1024, 1024, 512)


def c5_steps_torch(seed, shape, count, device, velocity=(1.5, 0.7, 0.3)):
    """Config 5's time steps on the device: step 0 is a k^-5/3 field plus a tanh front of width 4
    (amplitude 10x the std) and a zero slab over 10% of axis 0; step n is step 0 advected by n times
    the velocity (periodic trilinear resampling) plus white noise at 1e-3 of the range."""
    import torch
    base = grf_torch(seed, shape, 5.0 / 3.0, device)
    gen = np.random.default_rng(seed)
    nrm = gen.standard_normal(3)
    nrm /= np.linalg.norm(nrm)
    c = [gen.uniform(0.25 * s, 0.75 * s) for s in shape]
    ax = [torch.arange(s, device=device, dtype=torch.float32) for s in shape]
    d = (ax[0][:, None, None] - c[0]) * nrm[0] + (ax[1][None, :, None] - c[1]) * nrm[1] + (ax[2][None, None, :] - c[2]) * nrm[2]
    base += 10.0 * base.std() * torch.tanh(d / 4.0)
    del d
    z0 = int(gen.integers(0, shape[0] - shape[0] // 10))
    base[z0:z0 + shape[0] // 10] = 0.0
    g = torch.Generator(device=device).manual_seed(seed + 1)
    for n in range(count):
        if n == 0:
            yield base.clone()
            continue
        out = base
        for axis, v in enumerate(velocity):
            s = v * n
            i = int(np.floor(s))
            w = s - i
            out = (1 - w) * torch.roll(out, i, dims=axis) + w * torch.roll(out, i + 1, dims=axis)
        out += torch.randn(shape, generator=g, device=device) * (1e-3 * float(out.max() - out.min()))
        yield out.contiguous()


def series_section(ctx, dev, rank, steps=16, batch=4, rel_eb=1e-4):
    """Config 5: 16 steps of a 1024x1024x512 field (2 GiB each), REL 1e-4. Step 0: plan search and
    coefficient scan; steps 1-15: step 0's plan, gradient-tuned coefficients, 4 steps per batched
    call. Against full tuning of steps 1 and 15 on their own (plan search + scan)."""
    import time

    import torch

    from asz_b200 import api, series
    p = api.default_params(block_pivot_ratio=BPR)
    nbytes = 4 * C5_SHAPE[0] * C5_SHAPE[1] * C5_SHAPE[2]
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    out = []
    for s in series.compress_series(ctx, c5_steps_torch(500 + rank, C5_SHAPE, steps, dev), rel_eb, p, "cubic", batch):
        out.append({"index": s.index, "len": len(s.blob), "tune_ms": s.tune_ms, "call_s": s.info.get("call_s"),
                    "batch_total_s": s.info.get("batch_total_s"), "abs_eb": s.report.abs_eb})
    torch.cuda.synchronize(dev)
    total_s = time.perf_counter() - t0
    plan = None
    full = {}
    for k, x in enumerate(c5_steps_torch(500 + rank, C5_SHAPE, steps, dev)):
        if k not in (1, steps - 1):
            continue
        torch.cuda.synchronize(dev)
        t1 = time.perf_counter()
        blob, r = ctx.compress(x, rel_eb, None, "cubic", p)
        full[k] = {"len": len(blob), "call_s": time.perf_counter() - t1, "plan_s": r.plan_s, "plan": r.plan.decode()}
        plan = plan or r.plan.decode()
        del x
    later = [o for o in out if o["index"] > 0]
    batches_s = sum({o["batch_total_s"] for o in later})
    return {"steps": steps, "shape": "x".join(map(str, C5_SHAPE)), "bytes_per_step": nbytes, "rel_eb": rel_eb,
            "batch": batch, "total_s": total_s, "series_gbs": steps * nbytes / total_s / 1e9,
            "step0_full_tuning_s": out[0]["call_s"],
            "later_tune_ms_mean": sum(o["tune_ms"] for o in later) / len(later),
            "later_batched_calls_s": batches_s, "later_gbs": len(later) * nbytes / batches_s / 1e9,
            "cr": [nbytes / o["len"] for o in out],
            "full_tuning": {str(k): {**v, "cr": nbytes / v["len"],
                                     "cr_reuse_over_full": out[k]["len"] and v["len"] / out[k]["len"]}
                            for k, v in full.items()},
            "timing": "host wall clock; total_s covers generating the steps on the device, step 0's full tuning "
                      "and the later steps' tuning and batched calls (zstd included)"}


def batch_section(ctx, dev, rank, count=48, lo=96, hi=512, steps=3):
    """Config 3: 48 fields, dims U[96,512] per axis, alpha U[3,5], one plan (searched on field 0,
    reused for all) at REL 1e-3, block_pivot_ratio 3, cubic. Batched call against the fields
    compressed one call each; every field's bytes compared."""
    import time

    import torch

    from asz_b200 import api
    rng = np.random.default_rng(300 + rank)
    shapes = [tuple(int(v) for v in rng.integers(lo, hi + 1, size=3)) for _ in range(count)]
    alphas = rng.uniform(3, 5, size=count)
    xs = [grf_torch(3000 + 97 * rank + i, sh, float(a), dev) for i, (sh, a) in enumerate(zip(shapes, alphas))]
    total = sum(4 * x.numel() for x in xs)
    p = api.default_params(block_pivot_ratio=BPR)
    _, r0 = ctx.compress(xs[0], REL_EB, None, "cubic", p)
    plan = r0.plan.decode()
    blobs, _, br = ctx.compress_batch(xs, REL_EB, plan, "cubic", p)  # first call: autotuner + capture
    first = br.as_dict()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    rounds_ms = call_s = 0.0
    for _ in range(steps):
        blobs, _, br = ctx.compress_batch(xs, REL_EB, plan, "cubic", p)
        rounds_ms += br.rounds_ms
        call_s += br.total_s
    wall_s = (time.perf_counter() - t0) / steps
    batch_s = call_s / steps
    last = br.as_dict()
    single_s, exact = 0.0, 0
    for x, b in zip(xs, blobs):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        one, _ = ctx.compress(x, REL_EB, plan, "cubic", p)
        single_s += time.perf_counter() - t0
        exact += int(one == b)
    out_bytes = sum(len(b) for b in blobs)
    return {"fields": count, "dims": f"U[{lo},{hi}] per axis", "alpha": "U[3,5]", "input_bytes": total,
            "plan": plan, "plan_source": "plan search on field 0, reused for every field",
            "rel_eb": REL_EB, "cr": total / out_bytes, "bit_exact_fields": exact,
            "batch_call_s": batch_s, "batch_gbs": total / batch_s / 1e9, "batch_python_wall_s": wall_s,
            "rounds_device_ms": rounds_ms / steps, "rounds_gbs": total / (rounds_ms / steps / 1000) / 1e9,
            "single_calls_s": single_s, "single_gbs": total / single_s / 1e9, "speedup": single_s / batch_s,
            "first_call": {k: first[k] for k in ("total_s", "tune_s", "tuned_now")},
            "steady_call": {k: last[k] for k in ("total_s", "h2d_s", "prep_s", "rounds_s", "encode_s", "zstd_s",
                                                 "graph_reused", "fields_fallback", "fast_ctas_per_sm",
                                                 "round_ctas_per_sm", "tpl_shift", "kernel_launches")},
            "timing": "batch_call_s: the library's wall time of one batched C-ABI call (asz_batch_report.total_s), "
                      "inputs resident on the device, each field's .asz on the host (zstd included); "
                      "batch_python_wall_s adds the Python wrapper's copies of the 48 outputs; single_calls_s: host "
                      "wall clock around 48 asz_compress calls; rounds_device_ms: CUDA events around the captured "
                      "round sequence"}
def sweep_section(ctx, dev, rank, rel_eb=1e-3, with_reference=True, ref_planes=50):
    """The prediction sweep of s2_many_prediction on the C1 shape (100x500x500 k^-11/3 GRF + blobs
    + noise): all 27 predictors with the legacy grids and targets at one error bound (594 rows),
    the field resident on the device. Beside it, the reference tool (oracle/_ref, built from its
    sources) on the first `ref_planes` planes for the 1d4r2 stencil (39 rows), with our rows on the
    same slab compared line by line with its printed figures."""
    import torch

    from asz_b200 import fields
    from asz_b200 import sweep as sw
    x = fields.c1_field(seed=11 + rank, shape=C1_SHAPE)
    xd = torch.from_numpy(x).to(dev)
    preds = sw.predictors("all")
    sw.run(ctx, xd, preds[0], [rel_eb])
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    nrows = targets = 0
    enc = 0.0
    for p in preds:
        rows, _ = sw.run(ctx, xd, p, [rel_eb])
        nrows += len(rows)
        targets += sum(r.samples for r in rows)
        enc += sum(r.encode_seconds for r in rows)
    gpu_s = time.perf_counter() - t0
    out = {"field": "x".join(map(str, C1_SHAPE)) + " k^-11/3 GRF + 20 blobs + 1e-4 noise", "rel_eb": rel_eb,
           "predictors": len(preds), "rows": nrows, "targets": targets, "wall_s": gpu_s, "rows_per_s": nrows / gpu_s,
           "targets_per_s": targets / gpu_s, "encode_share": enc / gpu_s,
           "timing": "host wall clock around one asz_sweep call per predictor (field on the device): prediction, "
                     "histograms, Huffman encoding on the GPU, H1, framing and libzstd level 3 on the host threads; "
                     "encode_share: the part spent from the histograms to the last zstd"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    exe = O.ref_binary("s2_many_prediction")
    if with_reference and rank == 0 and exe is not None:
        slab = np.ascontiguousarray(x[:ref_planes])
        with tempfile.TemporaryDirectory() as wd:
            inp = os.path.join(wd, "slab.f32")
            slab.tofile(inp)
            t0 = time.perf_counter()
            r = subprocess.run([exe, inp, *map(str, slab.shape), os.path.join(wd, "ref"), "1d4r2", repr(rel_eb)],
                               capture_output=True, text=True)
            ref_s = time.perf_counter() - t0
        if r.returncode == 0:
            ref_lines = [ln for ln in r.stdout.splitlines() if not ln.startswith(("predictor=", "total_seconds="))]
            ours, ours_rows, t0 = [], 0, time.perf_counter()
            for p in sw.predictors("1d4r2"):
                rows, mm = sw.run(ctx, slab, p, [rel_eb])
                ours_rows += len(rows)
                for g in rows:
                    ours += [f"rel_eb={g.rel_eb:f}, t={g.c0:f}", f"BR={g.br:f}, CR={g.cr:f}", f"H1={g.h1:f}, H1_cr={g.h1_cr:f}",
                             f"RMSE={g.rmse:f}, MAE={g.mae:f}", f"PSNR={g.psnr:f}", ""]
            ours_s = time.perf_counter() - t0
            ref_rows = sum(1 for ln in ref_lines if ln.startswith("BR="))
            out["reference"] = {"sample": f"reference s2_many_prediction, stencil 1d4r2 (3 orders x 13 t) at {rel_eb:g} "
                                          f"on a {'x'.join(map(str, slab.shape))} slab, one core, wall time",
                                "kind": "reference", "cores": 1, "rows": ref_rows, "wall_s": ref_s,
                                "rows_per_s": ref_rows / ref_s, "ours_rows_per_s_same_slab": ours_rows / ours_s,
                                "speedup_same_slab": (ref_s / ref_rows) / (ours_s / ours_rows),
                                "printed_lines_identical": ours == ref_lines[3:]}
    return out


SELECTION_FAMILIES = ("tsel_fast", "tsel_exact", "tsel_serial")
GRAD_REPEATS = 7


def grad_tune_section(ctx, L, dev, rank, barrier):
    """Per-block t tuning on a C4-recipe field (256^3, per-octant anisotropy): the reference's
    candidate scan (the library's selection kernels inside a plain compression, device time) against
    the gradient tuner (open-loop gather + one tune launch, device time), with the resulting
    compression ratios and errors. Plan from the plan search, block_pivot_ratio 3."""
    import torch

    from asz_b200 import api, fields, grad
    x = torch.from_numpy(fields.c4_field(seed=4 + rank, shape=C4_SHAPE)).to(dev)
    entries = (PROFILE_ENTRY * 64)()
    out = {"field": "x".join(map(str, C4_SHAPE)) + " per-octant anisotropic GRF (corr. lengths U[2,64], slopes U[2.5,5])",
           "plan_source": "plan search (no plan given), block_pivot_ratio 3, cubic",
           "tuner": {"steps": grad.STEPS, "step0": grad.STEP0, "step_cap": grad.STEP_CAP}}

    def profiled(fn):
        L.asz_profile_enable(ctx._c, 1)
        L.asz_profile_read(ctx._c, entries, 64, 1)
        r = fn()
        n = L.asz_profile_read(ctx._c, entries, 64, 1)
        L.asz_profile_enable(ctx._c, 0)
        return r, {entries[i].name.decode(): entries[i].ms for i in range(min(n, 64))}

    for rel_eb in (1e-3, 1e-4):
        p = api.default_params(block_pivot_ratio=BPR)
        _, rep0 = ctx.compress(x, rel_eb, None, "cubic", p)
        plan = rep0.plan.decode()
        ctx.compress(x, rel_eb, plan, "cubic", p)  # warm-up
        barrier()
        # Repeats: the two sides are a few hundred microseconds and a few milliseconds of device
        # time, so the medians and the spread of REPEATS runs each are reported.
        plain_runs = []
        for _ in range(GRAD_REPEATS):
            (blob, rep), prof = profiled(lambda: ctx.compress(x, rel_eb, plan, "cubic", p))
            plain_runs.append(sum(prof.get(k, 0.0) for k in SELECTION_FAMILIES))
        plain_sel_ms = float(np.median(plain_runs))
        _, plain_psnr = ctx.stats()
        plain = {"selection_ms": plain_sel_ms, "cr": 4 * x.numel() / len(blob), "psnr_db": plain_psnr,
                 "exact_groups": int(rep.exact_groups)}
        ctx.set_tsel_mode(1)
        (_, _), prof1 = profiled(lambda: ctx.compress(x, rel_eb, plan, "cubic", p))
        ctx.set_tsel_mode(0)
        plain["selection_ms_exact_replay_everywhere"] = sum(prof1.get(k, 0.0) for k in SELECTION_FAMILIES)
        # Gradient tuner: gather + tune, device time (one untimed run first).
        grad_runs = []
        for k in range(GRAD_REPEATS + 1):
            prob, gprof = profiled(lambda: grad.prepare(ctx, x, rel_eb, plan, p))
            codes, info = grad.tune(prob)
            g_ms, t_ms = gprof.get("grad_gather", 0.0), info.pop("kernel_ms")
            if k:
                grad_runs.append((g_ms + t_ms, g_ms, t_ms))
        order = sorted(grad_runs)
        _, gather_ms, tune_ms = order[len(order) // 2]
        gblob, grep_ = ctx.compress_with_t(x, rel_eb, plan, "cubic", p, codes)
        gmax, gpsnr = ctx.stats()
        g = {"gather_ms": gather_ms, "tune_ms": tune_ms, "selection_ms": gather_ms + tune_ms,
             "cr": 4 * x.numel() / len(gblob), "psnr_db": gpsnr, "max_err_over_eb": gmax / grep_.abs_eb,
             "groups": prob.groups, "samples": int(prob.info.samples), **{k: v for k, v in info.items()}}
        sel = [r[0] for r in grad_runs]
        out[f"rel_eb_{rel_eb:g}"] = {
            "plan": plan, "plain_scan": plain, "gradient": g,
            "repeats": GRAD_REPEATS,
            "plain_scan_ms_range": [min(plain_runs), max(plain_runs)],
            "gradient_ms_range": [min(sel), max(sel)],
            "speedup_range": [min(plain_runs) / max(sel), max(plain_runs) / min(sel)],
            "speedup": plain_sel_ms / g["selection_ms"] if g["selection_ms"] else None,
            "speedup_vs_exact_replay": plain["selection_ms_exact_replay_everywhere"] / g["selection_ms"]
            if g["selection_ms"] else None,
            "cr_ratio": g["cr"] / plain["cr"]}
        del prob
    del x
    return out

# DRAM traffic per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the kernel families, from
# an ncu capture of a 256x512x512 C2 field (plan cubic2_012 x9, REL 1e-3): the mean per launch,
# doubled for the 512^3 field (the traffic grows with the number of values).
# huff_encode is one scope of two launches (tile bit counts, then packing) per compression.
TRAFFIC_PER_LAUNCH = {
    "tsel_fast": 2 * (292.08e6 + 31.40e6),
    "round_compress": 2 * (356.46e6 + 112.61e6),
    "round_decompress": 2 * (215.93e6 + 92.74e6),
    "huff_encode": 2 * (268.67e6 + 0.22e6 + 270.10e6 + 39.89e6),
}


# End-to-end calls in flight: on one GPU, twelve (measured: 4 -> 16.5, 8 -> 24.4, 12 -> 28.9,
# 16 -> 28.6 GB/s); with several ranks on one host, four per rank, so that the ranks' pinned
# buffers and host threads stay modest.
E2E_WORKERS = 12
E2E_WORKERS_PER_RANK = 4


def e2e_pipelined(api, L, local, dims, p, plan_b, xh, yh, blob, steps, barrier, workers):
    """`steps` compressions of the pinned host field xh and `steps` decompressions of `blob` into
    pinned host memory, `workers` calls in flight: each worker thread owns a context and takes
    the next step until all are done. Returns (compress ms, decompress ms), host wall clock with
    the device idle at both ends. Every call is the full C-ABI call (copies, kernels, libzstd)."""
    import threading
    import time

    import torch
    ctxs = [api.Context(local) for _ in range(workers)]
    blob_np = np.frombuffer(blob, dtype=np.uint8)
    outs = [torch.empty_like(yh).pin_memory() for _ in range(workers)]

    def comp(c):
        outp, outn, rep = _C.POINTER(_C.c_uint8)(), _C.c_size_t(0), api.Report()
        rc = L.asz_compress(c._c, _C.c_void_p(xh.data_ptr()), 0, dims, _C.c_float(REL_EB), _C.byref(p), plan_b,
                            _C.byref(outp), _C.byref(outn), _C.byref(rep))
        if rc:
            raise api.AszError(rc, L.asz_last_error(c._c).decode())
        L.asz_free(outp)

    def dec(c, out):
        rep = api.Report()
        rc = L.asz_decompress(c._c, _C.c_void_p(blob_np.ctypes.data), len(blob), dims, _C.c_float(REL_EB), _C.byref(p),
                              _C.c_void_p(out.data_ptr()), 0, _C.byref(rep))
        if rc:
            raise api.AszError(rc, L.asz_last_error(c._c).decode())

    def run(work):
        left = [steps]
        lock = threading.Lock()
        errs = []

        def worker(w):
            try:
                while True:
                    with lock:
                        if left[0] == 0:
                            return
                        left[0] -= 1
                    work(w)
            except Exception as e:  # noqa: BLE001 - re-raised below
                errs.append(e)

        ts = [threading.Thread(target=worker, args=(w,)) for w in range(workers)]
        barrier()
        t0 = time.perf_counter()
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3
        if errs:
            raise errs[0]
        return ms

    for w in range(workers):  # first call per context: its buffers
        comp(ctxs[w])
        dec(ctxs[w], outs[w])
    comp_ms = run(lambda w: comp(ctxs[w]))
    dec_ms = run(lambda w: dec(ctxs[w], outs[w]))
    for c in ctxs:
        c.close()
    return comp_ms, dec_ms


class PROFILE_ENTRY(_C.Structure):
    _fields_ = [("name", _C.c_char * 32), ("launches", _C.c_uint64), ("ms", _C.c_double), ("bytes", _C.c_uint64)]


if __name__ == "__main__":
    main()
