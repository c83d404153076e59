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
