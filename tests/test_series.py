"""Time series with plan reuse: step 0 fully tuned, later steps with step 0's plan and gradient-tuned
coefficients, compressed in batches. Each later stream must equal the oracle's compression of that
step with the same plan and codes, and decode within the error bound."""
import os
import tempfile

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _steps(n, shape=(48, 40, 56)):
    from asz_b200 import fields
    return [fields.c5_step(k, seed=5, shape=shape) for k in range(n)]


def test_series_plan_reuse(gpu_ctx):
    import asz_b200.api as api
    from asz_b200 import plans, series
    xs = _steps(6)
    p = api.default_params(block_pivot_ratio=3)
    with tempfile.TemporaryDirectory() as d:
        pf = os.path.join(d, "plans.json")
        out = list(series.compress_series(gpu_ctx, xs, 1e-4, p, "cubic", batch=2, plan_file=pf))
        plan = out[0].info["plan"]
        assert plans.for_rel_eb(plans.load(pf), 1e-4)[0] == plan.split(",")
    assert [s.index for s in out] == list(range(6))
    full0, _ = gpu_ctx.compress(xs[0], 1e-4, None, "cubic", p)
    assert out[0].blob == full0
    op = O.default_params(block_pivot_ratio=3)
    for s in out[1:]:
        codes = s.info["codes"].cpu().numpy()
        o = O.compress(xs[s.index], 1e-4, plan, False, op, t_int=codes)
        assert s.blob == o.asz
        dec = O.decompress(s.blob, xs[s.index].shape, 1e-4, op)
        assert np.abs(dec.astype(np.float64) - xs[s.index]).max() <= 1.01 * o.abs_eb
        full, _ = gpu_ctx.compress(xs[s.index], 1e-4, None, "cubic", p)
        assert len(s.blob) <= 1.05 * len(full)  # plan reused, coefficients tuned: close to a full search
