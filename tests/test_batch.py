"""Batched compression: many fields of uneven shapes with one plan and one error bound. Every
field's .asz must equal its single-field compression (itself checked against the oracle), with
the launch-shape autotuner's first call and the captured round sequence's replay."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _fields(seed, count, lo, hi):
    from asz_b200 import fields
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        shape = tuple(int(x) for x in rng.integers(lo, hi + 1, size=3))
        f = fields.grf_field(shape, rng.uniform(3, 5), rng).astype(np.float32)
        if i % 5 == 4:
            f = f + rng.random(shape).astype(np.float32) * 0.5  # noisy: groups for the exact path
        out.append(f)
    return out


@pytest.mark.parametrize("plan,family", [(",".join(["cubic0_012", "cubic1_012", "cubic2_012"] * 3), "cubic"),
                                         (",".join(["cubic2_012"] * 5), "quintic")])
def test_batch_equals_single_field(gpu_ctx, plan, family):
    import asz_b200.api as api
    fs = _fields(7 if family == "cubic" else 8, 9, 12, 70)
    p = api.default_params(block_pivot_ratio=3)
    for call in range(2):  # first call tunes and captures, second replays the graph
        blobs, reps, br = gpu_ctx.compress_batch(fs, 1e-3, plan, family, p)
        assert br.graph_reused == (1 if call else 0)
        assert br.tuned_now == (0 if call else 1)
        for f, blob in zip(fs, blobs):
            single, _ = gpu_ctx.compress(f, 1e-3, plan, family, p)
            assert blob == single
    o = O.compress(fs[0], 1e-3, plan, family == "quintic", O.default_params(block_pivot_ratio=3))
    assert blobs[0] == o.asz
    # New data of the same shapes replays the captured sequence: the values it reads (error
    # bounds, slopes, classes) come from the fields' records, not from the capture.
    fs2 = [f * 3.0 + 1.0 for f in fs]
    blobs2, _, br2 = gpu_ctx.compress_batch(fs2, 1e-3, plan, family, p)
    assert br2.graph_reused == 1
    for f, blob in zip(fs2, blobs2):
        single, _ = gpu_ctx.compress(f, 1e-3, plan, family, p)
        assert blob == single


def test_batch_groups_beyond_shared_memory(gpu_ctx):
    """Groups of more samples than the exact kernel's shared memory holds (24^3 blocks sampled
    2048 at a time, so the finest rounds' groups run to thousands of samples; noisy fields, so
    many of them reach the exact path): the batched sequence replays those in global scratch, a
    CTA per group, and every field's bytes equal its single-field compression and the oracle's."""
    import asz_b200.api as api
    from asz_b200 import fields
    rng = np.random.default_rng(43)
    fs = []
    for _ in range(3):
        shape = tuple(int(x) for x in rng.integers(60, 76, size=3))
        fs.append(fields.grf_field(shape, 4.0, rng).astype(np.float32) + rng.random(shape).astype(np.float32) * 0.5)
    plan = ",".join(["cubic0_012", "cubic1_012", "cubic2_012"] * 2)
    p = api.default_params(block_pivot_ratio=6, h1_block_sampling_num=2048)
    blobs, _, _ = gpu_ctx.compress_batch(fs, 1e-4, plan, "cubic", p)
    handed_off = 0
    for f, blob in zip(fs, blobs):
        single, rep = gpu_ctx.compress(f, 1e-4, plan, "cubic", p)
        assert blob == single
        handed_off += rep.exact_groups
    assert handed_off > 0
    o = O.compress(fs[0], 1e-4, plan, False, O.default_params(block_pivot_ratio=6, h1_block_sampling_num=2048))
    assert blobs[0] == o.asz


def test_batch_device_inputs_and_errors(gpu_ctx):
    import torch

    import asz_b200.api as api
    fs = _fields(11, 5, 20, 60)
    plan = ",".join(["cubic0_012", "cubic1_012", "cubic2_012"] * 2)
    p = api.default_params(block_pivot_ratio=4)
    dev = [torch.from_numpy(f).cuda() for f in fs]
    blobs, reps, br = gpu_ctx.compress_batch(dev, 1e-4, plan, "cubic", p)
    for f, blob, r in zip(fs, blobs, reps):
        single, sr = gpu_ctx.compress(f, 1e-4, plan, "cubic", p)
        assert blob == single
        assert r.abs_eb == sr.abs_eb and r.default_slope == sr.default_slope
        dec, _ = gpu_ctx.decompress(blob, f.shape, 1e-4, p)
        assert np.abs(dec.astype(np.float64) - f).max() <= 1.01 * r.abs_eb
    bad = fs[:2] + [np.zeros((10, 10, 10), np.float32)]
    with pytest.raises(api.AszError, match="field 2: max_val==min_val"):
        gpu_ctx.compress_batch(bad, 1e-3, plan, "cubic", p)
