"""The 8-wide BVH build (MRT_BVH_WIDE) on the host (no GPU): structure and
conservative quantised boxes, over random, degenerate and full-size inputs.

mrt_bvh_build_check builds the wide tree and checks that every node is
reached once, every primitive sits in one leaf, and every 8-bit slot box
contains the primitive boxes below it (the property that keeps culling from
dropping a hit the binary tree or the reference would find)."""
import numpy as np
import pytest

import mrt
import scenes


def boxes_of(mn, mx):
    return np.concatenate([mn, mx], 1)


def random_boxes(rng, n, scale=10.0, size=0.5):
    c = rng.uniform(-scale, scale, (n, 3))
    h = rng.uniform(0.0, size, (n, 3))
    return boxes_of(c - h, c + h)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 8, 9, 33, 100, 10000])
def test_random_boxes(n):
    rng = np.random.default_rng(n)
    st = mrt.bvh_build_check(random_boxes(rng, n))
    assert st["wide"] and st["nodes"] >= 1 and -(-n // 4) <= st["leaves"] <= n


def test_identical_boxes():
    b = np.tile([[-1.0, -1.0, -1.0, 1.0, 1.0, 1.0]], (1000, 1))
    assert mrt.bvh_build_check(b)["wide"]


def test_flat_and_point_boxes():
    rng = np.random.default_rng(7)
    # a wall of triangles at x = -25 exactly (zero extent on x), and points
    c = rng.uniform(-5, 5, (4000, 3))
    c[:2000, 0] = -25.0
    h = rng.uniform(0, 0.2, (4000, 3))
    h[:2000, 0] = 0.0
    h[2000:] = 0.0
    assert mrt.bvh_build_check(boxes_of(c - h, c + h))["wide"]


@pytest.mark.parametrize("offset,size", [(1e6, 1e-3), (1e-6, 1e-9), (1e30, 1e24), (-3e4, 1e-2)])
def test_far_and_tiny_boxes(offset, size):
    rng = np.random.default_rng(3)
    c = offset + rng.uniform(-size * 100, size * 100, (2000, 3))
    h = rng.uniform(0, size, (2000, 3))
    assert mrt.bvh_build_check(boxes_of(c - h, c + h))["wide"]


def test_binary_option_still_builds():
    rng = np.random.default_rng(11)
    st = mrt.bvh_build_check(random_boxes(rng, 5000), mode=mrt.BVH_SAH)
    assert not st["wide"] and st["leaves"] >= 5000 // 8


def test_c1_mesh():
    """c1's 1,310,720-triangle displaced sphere: wide tree with depth and
    node count in the expected range."""
    sc = scenes.CONFIGS["c1"]()
    m = sc.meshes[0]
    tris = m.positions[m.indices]
    mn, mx = tris.min(axis=1), tris.max(axis=1)
    st = mrt.bvh_build_check(boxes_of(mn, mx))
    n = len(tris)
    assert st["wide"] and n / 4 <= st["leaves"] <= n
    assert st["depth"] <= 16
    # nodes well filled: (internal + leaf slots) / nodes above 6 of 8
    assert (st["nodes"] - 1 + st["leaves"]) / st["nodes"] > 6.0
    assert n / 32 <= st["nodes"] <= n / 8
