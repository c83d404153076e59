"""The differentiable coefficient tuner: the relaxed proxy's gradient (float64 torch restatement
against central finite differences on the CPU; the CUDA forward and backward kernels against the
float64 restatement), the open-loop samples against the oracle, and tuned streams against the
oracle and the reference's decoder semantics."""
import numpy as np
import pytest
import torch

import oracle as O
from asz_b200.grad import BINS, HALF_BINS, relaxed_proxy_torch


def _synthetic_problem(rng, groups=60, per=(20, 400)):
    n = rng.integers(per[0], per[1], size=groups)
    n[::7] = 0  # groups without samples
    off = np.concatenate([[0], np.cumsum(n)]).astype(np.int64)
    S = int(off[-1])
    eb = rng.uniform(1e-3, 1e-2, size=groups)
    A = rng.normal(0, 1, S) * np.repeat(rng.uniform(0.002, 0.2, groups), n)
    B = rng.normal(0, 1, S) * np.repeat(rng.uniform(0.001, 0.05, groups), n)
    meta = np.stack([eb, 0.2 * eb, 0.5 / (0.2 * eb), rng.uniform(1, 30, groups)], 1)
    return A, B, off, meta


def test_relaxed_proxy_gradient_matches_central_differences():
    """float64: autograd of the restated proxy equals central differences (h = 1e-7) wherever no
    sample's bin changes inside [t - h, t + h]; relative error below 1e-6."""
    rng = np.random.default_rng(11)
    A, B, off, meta = _synthetic_problem(rng)
    At, Bt = torch.tensor(A), torch.tensor(B)
    offt, metat = torch.tensor(off), torch.tensor(meta)
    G = len(off) - 1
    R2 = 4.0
    t = torch.tensor(rng.uniform(0.07, 0.37, G), requires_grad=True)
    J = relaxed_proxy_torch(At, Bt, offt, metat, R2, t)
    J.sum().backward()
    g = t.grad.numpy()
    h = 1e-7
    with torch.no_grad():
        Jp = relaxed_proxy_torch(At, Bt, offt, metat, R2, t + h).numpy()
        Jm = relaxed_proxy_torch(At, Bt, offt, metat, R2, t - h).numpy()
    fd = (Jp - Jm) / (2 * h)
    n = np.diff(off)
    seg = np.repeat(np.arange(G), n)
    tt = t.detach().numpy()
    checked = 0
    for gi in range(G):
        if n[gi] == 0:
            assert g[gi] == 0.0 and J[gi].item() == 0.0
            continue
        s = seg == gi
        q = lambda tv: np.clip((A[s] * tv + B[s]) / (2 * meta[gi, 0]), -HALF_BINS, HALF_BINS)
        if not np.array_equal(np.floor(q(tt[gi] - h)), np.floor(q(tt[gi] + h))):
            continue
        checked += 1
        assert abs(g[gi] - fd[gi]) <= 1e-6 * max(abs(fd[gi]), 1e-3), (gi, g[gi], fd[gi])
    assert checked > G // 2
    assert BINS == 2 * HALF_BINS + 2


# ---------------------------------------------------------------------------------------------
# GPU


def _c4_small(seed=4, shape=(64, 64, 64)):
    from asz_b200 import fields
    return fields.c4_field(seed=seed, shape=shape)


@pytest.mark.gpu
def test_gather_matches_oracle(gpu_ctx):
    """The device gather of open-loop samples equals the oracle's restatement bit for bit."""
    import asz_b200.api as api
    from asz_b200 import fields, grad
    rng = np.random.default_rng(5)
    orders = ["120", "021", "012"]
    for i in range(8):
        shape = tuple(int(x) for x in rng.integers(12, 60, size=3))
        f = fields.grf_field(shape, rng.uniform(1.5, 5), rng).astype(np.float32)
        plan = ",".join(f"cubic{rng.integers(0, 3)}_{orders[rng.integers(0, 3)]}" for _ in range(int(rng.integers(2, 9))))
        bpr = int(rng.integers(2, 6))
        eb = float(10 ** rng.uniform(-4, -2))
        prob = grad.prepare(gpu_ctx, f, eb, plan, api.default_params(block_pivot_ratio=bpr))
        A, B, off = O.grad_samples(f, eb, plan, O.default_params(block_pivot_ratio=bpr))
        assert np.array_equal(prob.offsets.cpu().numpy().astype(np.uint64), off)
        assert np.array_equal(prob.A.cpu().numpy().view(np.uint32), A.view(np.uint32))
        assert np.array_equal(prob.B.cpu().numpy().view(np.uint32), B.view(np.uint32))


def _problem(gpu_ctx, rel_eb=1e-3):
    import asz_b200.api as api
    from asz_b200 import grad
    f = _c4_small()
    p = api.default_params(block_pivot_ratio=3)
    _, rep = gpu_ctx.compress(f, rel_eb, None, "cubic", p)
    plan = rep.plan.decode()
    return f, plan, p, grad.prepare(gpu_ctx, torch.from_numpy(f).cuda(), rel_eb, plan, p)


@pytest.mark.gpu
def test_forward_and_backward_kernels_match_fp64(gpu_ctx):
    """FP32 kernels against the float64 restatement on a C4-recipe field: J within 1e-5 relative
    (median) and 1e-3 (worst); dJ/dt within 1e-3 relative (median) and 5e-2 for 99% of groups. The
    kernel rounds q in float and sums soft-bin weights in fixed point (2^-24 per unit), so a sample
    within float rounding of a bin edge can move one unit of weight; that is the tail."""
    from asz_b200.grad import RelaxedProxy
    f, plan, p, prob = _problem(gpu_ctx)
    G = prob.groups
    rng = np.random.default_rng(3)
    t = torch.tensor(rng.uniform(0.07, 0.37, G), dtype=torch.float32, device="cuda").requires_grad_(True)
    J = RelaxedProxy.apply(t, prob)
    gJ = torch.tensor(rng.uniform(0.5, 2.0, G), dtype=torch.float32, device="cuda")
    (J * gJ).sum().backward()
    t64 = t.detach().double().requires_grad_(True)
    J64 = relaxed_proxy_torch(prob.A.double(), prob.B.double(), prob.offsets, prob.meta.double(), float(prob.info.R2), t64)
    (J64 * gJ.double()).sum().backward()
    n = torch.diff(prob.offsets.long()).cpu().numpy()
    live = n > 0
    J32, J64n = J.detach().cpu().double().numpy()[live], J64.detach().cpu().numpy()[live]
    rj = np.abs(J32 - J64n) / np.maximum(np.abs(J64n), 1e-6)
    g32, g64 = t.grad.cpu().double().numpy()[live], t64.grad.cpu().numpy()[live]
    scale = np.maximum(np.abs(g64), 1e-3 * np.abs(g64).max())
    rg = np.abs(g32 - g64) / scale
    print(f"groups {live.sum()}: J rel err median {np.median(rj):.2e} max {rj.max():.2e}; "
          f"dJ/dt rel err median {np.median(rg):.2e} p99 {np.quantile(rg, 0.99):.2e}")
    assert np.median(rj) < 1e-5 and rj.max() < 1e-3
    assert np.median(rg) < 1e-3 and np.quantile(rg, 0.99) < 5e-2


@pytest.mark.gpu
def test_fused_tuner_follows_autograd_steps(gpu_ctx):
    """The one-launch tuner takes the same projected steps as the Python loop over the autograd
    function for the groups whose samples all fit its steps (1024; identical t for at least 99% of
    them; a gradient within rounding of zero may take the other sign)."""
    from asz_b200 import grad
    f, plan, p, prob = _problem(gpu_ctx)
    n = torch.diff(prob.offsets.long())
    codes, info = grad.tune(prob, with_relaxed=True, step_cap=1024)  # every sample up to 1024
    t_loop = grad.tune_with_autograd(prob)
    whole = n <= 1024
    assert whole.sum() >= 0.9 * len(n)
    same = (info["t_relaxed"] == t_loop)[whole].float().mean().item()
    assert same >= 0.99, same
    assert info["tuned"] == prob.groups - int((torch.diff(prob.offsets.long()) == 0).sum())


@pytest.mark.gpu
@pytest.mark.parametrize("rel_eb", [1e-3, 1e-4])
def test_tuned_stream_matches_oracle(gpu_ctx, rel_eb):
    """Tuned codes -> asz_compress_with_t: the same bytes as the oracle given the same codes, a
    reconstruction its decoder reproduces, max error within the reference's 1.01 eb, and a
    compression ratio within 2% of the full candidate scan on this 64^3 field."""
    from asz_b200 import grad
    f, plan, p, prob = _problem(gpu_ctx, rel_eb)
    codes, info = grad.tune(prob)
    codes = codes.cpu().numpy()
    blob, rep = gpu_ctx.compress_with_t(f, rel_eb, plan, "cubic", p, codes)
    o = O.compress(f, rel_eb, plan, False, O.default_params(block_pivot_ratio=3), t_int=codes)
    assert blob == o.asz
    assert np.array_equal(gpu_ctx.debug_t(), codes)
    dec, _ = gpu_ctx.decompress(blob, f.shape, rel_eb, p)
    assert np.array_equal(dec.view(np.uint32), o.recon.view(np.uint32))
    assert np.abs(dec.astype(np.float64) - f).max() <= 1.01 * o.abs_eb
    plain, prep = gpu_ctx.compress(f, rel_eb, plan, "cubic", p)
    print(f"rel_eb {rel_eb}: CR tuned {len(f.tobytes()) / len(blob):.4f} plain {len(f.tobytes()) / len(plain):.4f}; "
          f"{info}")
    assert len(blob) <= 1.02 * len(plain)


@pytest.mark.gpu
def test_given_t_errors(gpu_ctx):
    """Given t tables: a wrong length and a code outside [t_min, t_max] are rejected with a message;
    the tuner's launch rejects a team size it cannot run."""
    import ctypes as C

    import asz_b200.api as api
    from asz_b200 import grad
    f = _c4_small(shape=(40, 40, 48))
    plan = ",".join(["cubic0_012", "cubic1_012", "cubic2_012"] * 2)
    p = api.default_params(block_pivot_ratio=3)
    _, rep = gpu_ctx.compress(f, 1e-3, plan, "cubic", p)
    n = gpu_ctx.debug_t().size
    with pytest.raises(api.AszError, match="t table length"):
        gpu_ctx.compress_with_t(f, 1e-3, plan, "cubic", p, np.full(n + 1, 8, np.int64))
    with pytest.raises(api.AszError, match="outside"):
        gpu_ctx.compress_with_t(f, 1e-3, plan, "cubic", p, np.full(n, 13, np.int64))
    with pytest.raises(api.AszError, match="t table length"):
        gpu_ctx.compress_batch([f, f], 1e-3, plan, "cubic", p, t_tables=[np.full(n, 8, np.int64), np.full(3, 8, np.int64)])
    prob = grad.prepare(gpu_ctx, f, 1e-3, plan, p)
    assert prob.info.samples > 0
    with pytest.raises(api.AszError):
        grad.tune(prob, team=1024)
    codes, info = grad.tune(prob, team=64)
    blob, _ = gpu_ctx.compress_with_t(f, 1e-3, plan, "cubic", p, codes)
    o = O.compress(f, 1e-3, plan, False, O.default_params(block_pivot_ratio=3), t_int=codes.cpu().numpy())
    assert blob == o.asz
    # A plan whose every group falls back has no samples at all: every code stays the default.
    empty = grad.prepare(gpu_ctx, f[:8, :8, :8].copy(), 1e-3, "cubic0_012", api.default_params(block_pivot_ratio=2))
    assert empty.info.samples == 0
    codes0, _ = grad.tune(empty)
    assert (codes0 == 8).all()
