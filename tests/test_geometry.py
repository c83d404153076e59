"""Host-side check of the round kernels' target geometry (no GPU): bounds, read-after-write order
between rounds and the reference's QB layout, for random shapes, plans and block ratios."""
import ctypes as C

import numpy as np
import pytest

import asz_b200.api as api


def _check(dims, plan, bpr, quintic):
    L = api.lib()
    L.asz_check_geometry.argtypes = [C.POINTER(C.c_uint64), C.c_char_p, C.c_uint64, C.c_int]
    L.asz_check_geometry.restype = C.c_int64
    return L.asz_check_geometry((C.c_uint64 * 3)(*dims), plan.encode(), bpr, int(quintic))


def test_geometry_random_plans():
    rng = np.random.default_rng(11)
    orders = ["120", "021", "012"]
    for _ in range(150):
        dims = [int(x) for x in rng.integers(7, 50, size=3)]
        plan = ",".join(f"cubic{rng.integers(0, 3)}_{orders[rng.integers(0, 3)]}" for _ in range(int(rng.integers(1, 11))))
        assert _check(dims, plan, int(rng.integers(1, 6)), rng.integers(0, 2)) == 0, (dims, plan)


@pytest.mark.parametrize("dims,plan,bpr", [
    ((96, 96, 96), ",".join(["cubic2_012"] * 7), 3),
    ((100, 64, 72), ",".join(["cubic0_012", "cubic1_012", "cubic2_012"] * 3), 3),
    ((7, 7, 7), "cubic0_120,cubic1_021,cubic2_012", 1),
])
def test_geometry_named(dims, plan, bpr):
    assert _check(dims, plan, bpr, True) == 0
    assert _check(dims, plan, bpr, False) == 0


def _check_frame(dims, origin, plan, bpr, quintic):
    L = api.lib()
    L.asz_check_geometry_frame.argtypes = [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_char_p, C.c_uint64, C.c_int]
    L.asz_check_geometry_frame.restype = C.c_int64
    return L.asz_check_geometry_frame((C.c_uint64 * 3)(*dims), (C.c_uint64 * 3)(*origin), plan.encode(), bpr, int(quintic))


def test_geometry_frames():
    """Frames with a halo before the origin, as the predictor-family probe builds them: a context of
    one or two blocks per axis after up to 5 half pivot strides of halo."""
    rng = np.random.default_rng(12)
    orders = ["120", "021", "012"]
    for _ in range(200):
        plan = [f"cubic{rng.integers(0, 3)}_{orders[rng.integers(0, 3)]}" for _ in range(int(rng.integers(1, 7)))]
        ps = [1, 1, 1]
        for pr in plan:
            ps[int(pr[5])] *= 2
        bpr = int(rng.integers(1, 5))
        dims, origin = [], []
        for a in range(3):
            # predictor_family.tpp:40-50: the context starts at a block boundary (0 or more blocks in),
            # the halo is min(5 * (ps / 2), context start), the context spans 1 or 2 blocks (+ face).
            shape = ps[a] * bpr
            begin = shape * int(rng.integers(0, 4))
            halo = min(5 * (ps[a] // 2), begin)
            nblk = int(rng.integers(1, 3))
            span = nblk * shape + 1 if rng.random() < 0.7 else int(rng.integers(1, nblk * shape + 1))
            dims.append(halo + span)
            origin.append(halo)
        if min(dims) < 1:
            continue
        assert _check_frame(dims, origin, ",".join(plan), bpr, rng.integers(0, 2)) == 0, (dims, origin, plan, bpr)
