"""The host binned-SAH hierarchy builder (ordinarylight_b200/csrc/olc_sah.h),
compiled for the CPU with tests/sah_harness.cpp: every tree it returns is a
valid one-primitive-per-leaf BVH2 (each primitive in exactly one leaf, each
node's primitives a contiguous range of sorted positions, child boxes the
exact unions of their primitives' boxes), also for coincident, denormal-close
and non-finite centroids, and its summed inner-node area is below that of an
object-median tree."""

from __future__ import annotations

import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent / "ordinarylight_b200" / "csrc"


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ is not available")
    out = tmp_path_factory.mktemp("sah") / "libsah.so"
    subprocess.run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-I", str(CSRC), str(HERE / "sah_harness.cpp"),
                    "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    lib.sah_build_flat.restype = ctypes.c_int
    return lib


def _build(lib, lo, hi):
    lo = np.ascontiguousarray(lo, np.float32)
    hi = np.ascontiguousarray(hi, np.float32)
    with np.errstate(invalid="ignore"):   # -inf + inf in the non-finite case
        centre = np.ascontiguousarray((lo + hi) * np.float32(0.5), np.float32)
    n = len(lo)
    child = np.zeros((max(n - 1, 1), 2), np.int32)
    boxes = np.zeros((max(n - 1, 1), 2, 6), np.float32)
    order = np.zeros(n, np.uint32)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    m = lib.sah_build_flat(ctypes.c_uint32(n), p(lo), p(hi), p(centre), p(child), p(boxes), p(order))
    return m, child[:m], boxes[:m], order


def _check_tree(lo, hi, m, child, boxes, order):
    """Walk from the root: returns the summed inner-node box area."""
    n = len(lo)
    assert m == n - 1
    assert sorted(order.tolist()) == list(range(n))
    seen_nodes = np.zeros(m, bool)
    seen_leaves = np.zeros(n, bool)
    area = 0.0

    def visit(node):
        nonlocal area
        assert not seen_nodes[node]
        seen_nodes[node] = True
        ranges = []
        for s in range(2):
            c = int(child[node, s])
            if c >= 0:
                assert c > node            # children are created after their parent
                r = visit(c)
            else:
                k = ~c
                assert not seen_leaves[k]
                seen_leaves[k] = True
                r = (k, k + 1)
            prims = order[r[0]:r[1]]
            want_lo = lo[prims].min(axis=0)
            want_hi = hi[prims].max(axis=0)
            np.testing.assert_array_equal(boxes[node, s, :3], want_lo)
            np.testing.assert_array_equal(boxes[node, s, 3:], want_hi)
            ranges.append(r)
        assert ranges[0][1] == ranges[1][0]   # contiguous sorted positions
        blo = np.minimum(boxes[node, 0, :3], boxes[node, 1, :3]).astype(np.float64)
        bhi = np.maximum(boxes[node, 0, 3:], boxes[node, 1, 3:]).astype(np.float64)
        e = np.maximum(bhi - blo, 0.0)
        area += 2.0 * (e[0] * e[1] + e[1] * e[2] + e[2] * e[0])
        return (ranges[0][0], ranges[1][1])

    if n >= 2:
        assert visit(0) == (0, n)
        assert seen_nodes.all() and seen_leaves.all()
    return area


def _median_tree_area(lo, hi, idx):
    """Summed inner-node area of an object-median tree (largest centroid axis)."""
    if len(idx) < 2:
        return 0.0
    blo = lo[idx].min(axis=0).astype(np.float64)
    bhi = hi[idx].max(axis=0).astype(np.float64)
    e = bhi - blo
    own = 2.0 * (e[0] * e[1] + e[1] * e[2] + e[2] * e[0])
    c = (lo[idx] + hi[idx]) * 0.5
    axis = int(np.argmax(c.max(axis=0) - c.min(axis=0)))
    srt = idx[np.argsort(c[:, axis], kind="stable")]
    h = len(srt) // 2
    return own + _median_tree_area(lo, hi, srt[:h]) + _median_tree_area(lo, hi, srt[h:])


def _triangle_boxes(rng, n, spread=10.0, size=0.3):
    v0 = rng.uniform(-spread, spread, (n, 3))
    tri = v0[:, None, :] + rng.normal(scale=size, size=(n, 3, 3))
    return tri.min(axis=1).astype(np.float32), tri.max(axis=1).astype(np.float32)


@pytest.mark.parametrize("n", [2, 3, 5, 17, 64, 1000, 4096])
def test_random_triangles_give_a_valid_tree(harness, n):
    lo, hi = _triangle_boxes(np.random.default_rng(n), n)
    _check_tree(lo, hi, *_build(harness, lo, hi))


def test_clustered_primitives_cost_less_than_an_object_median_tree(harness):
    rng = np.random.default_rng(3)
    parts = [_triangle_boxes(rng, 3000, spread=2.0), _triangle_boxes(rng, 300, spread=40.0)]
    parts[0] = (parts[0][0] + np.float32(30.0), parts[0][1] + np.float32(30.0))
    lo = np.concatenate([p[0] for p in parts])
    hi = np.concatenate([p[1] for p in parts])
    sah_area = _check_tree(lo, hi, *_build(harness, lo, hi))
    median_area = _median_tree_area(lo, hi, np.arange(len(lo)))
    assert sah_area < 0.95 * median_area


def test_coincident_centroids_split_at_the_median(harness):
    n = 37
    lo = np.tile(np.float32([-1, -1, -1]), (n, 1))
    hi = np.tile(np.float32([1, 1, 1]), (n, 1))
    m, child, boxes, order = _build(harness, lo, hi)
    _check_tree(lo, hi, m, child, boxes, order)
    # the root's children hold 18 and 19 primitives
    sizes = []
    for s in range(2):
        c = int(child[0, s])
        stack, count = [c], 0
        while stack:
            x = stack.pop()
            if x < 0:
                count += 1
            else:
                stack.extend(int(v) for v in child[x])
        sizes.append(count)
    assert sizes == [18, 19]


def test_denormal_close_and_non_finite_centroids_stay_in_bounds(harness):
    n = 40
    tiny = np.float32(1e-44)
    lo = np.zeros((n, 3), np.float32)
    lo[:, 0] = np.arange(n, dtype=np.float32) * tiny   # extent so small that 16 / extent overflows
    hi = lo.copy()
    _check_tree(lo, hi, *_build(harness, lo, hi))
    lo2, hi2 = _triangle_boxes(np.random.default_rng(5), n)
    lo2[3] = -np.inf
    hi2[3] = np.inf
    lo2[7, 1] = np.nan
    m, child, boxes, order = _build(harness, lo2, hi2)
    assert m == n - 1 and sorted(order.tolist()) == list(range(n))
