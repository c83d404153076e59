"""Time series with plan reuse: full tuning on the first step, the plan reused for the later steps
with their per-block coefficients from the gradient tuner, compressed in batches.

The reference tunes every file on its own: the plan search (generate_config.tpp:444-678) and the
per-block coefficient scan (compress.tpp:91-144). Here the first step gets both; its plan is
recorded (optionally in a launcher plan file, asz_b200.plans) and every later step keeps that plan
while the gradient tuner (asz_b200.grad) chooses its coefficients, several steps to one batched
call (asz_compress_batch_with_t). Every stream is an ordinary .asz.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

from . import api, grad, plans


@dataclass
class SeriesStep:
    index: int
    blob: bytes
    report: object
    tune_ms: float = 0.0             # gather + tune device time (later steps)
    info: dict = field(default_factory=dict)


def compress_series(ctx: api.Context, steps, rel_eb: float, params: api.Params | None = None, family: str = "cubic",
                    batch: int = 4, plan_file=None):
    """Yield a SeriesStep per input step (torch CUDA tensors or NumPy arrays, all the same shape).

    Step 0: plan search and coefficient scan (ctx.compress with no plan). Later steps: the plan of
    step 0, coefficients from grad.tune, `batch` steps per batched call."""
    p = params if params is not None else api.default_params()
    it = iter(steps)
    x0 = next(it)
    t0 = time.perf_counter()
    blob0, rep0 = ctx.compress(x0, rel_eb, None, family, p)
    plan = rep0.plan.decode()
    if plan_file is not None:
        plans.record_plan(plan_file, rel_eb, rep0)
    yield SeriesStep(0, blob0, rep0, info={"plan": plan, "call_s": time.perf_counter() - t0})
    pending, index = [], 1

    def flush():
        codes, tune_ms, infos = [], [], []
        for x in pending:
            prob = grad.prepare(ctx, x, rel_eb, plan, p)
            c, info = grad.tune(prob)
            codes.append(c)
            tune_ms.append(info.pop("kernel_ms"))
            infos.append(info)
            del prob
        t1 = time.perf_counter()
        blobs, reps, br = ctx.compress_batch(pending, rel_eb, plan, family, p, t_tables=codes)
        call_s = time.perf_counter() - t1
        out = []
        for k, (b, r) in enumerate(zip(blobs, reps)):
            out.append(SeriesStep(index - len(pending) + k, b, r, tune_ms[k],
                                  {**infos[k], "batch_call_s": call_s, "batch_size": len(pending),
                                   "batch_total_s": br.total_s, "codes": codes[k]}))
        return out

    for x in it:
        pending.append(x)
        index += 1
        if len(pending) == batch:
            yield from flush()
            pending = []
    if pending:
        yield from flush()
