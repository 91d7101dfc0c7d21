"""Batched workload generator and configuration menu (CPU)."""
from ots import batch as B


def test_workload_is_seeded_and_in_range():
    a, b = B.workload(256, 2012), B.workload(256, 2012)
    assert a == b and len(a) == 256
    assert {g["stencil"] for g in a} == set(B.BATCH_STENCILS)
    assert all(64 <= g["n"] <= 2048 and 8 <= g["steps"] <= 256 for g in a)
    assert B.workload(256, 1) != a


def test_menu_covers_the_instantiated_shapes():
    assert len(B.MENU) == 8 * 3 * 3
    assert {m["bx"] for m in B.MENU} == {16, 32, 64}
    assert {m["E"] for m in B.MENU} == {1, 2, 4}
