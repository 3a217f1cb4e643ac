"""ORACLE — test infrastructure only, never part of the product path.

Host restatement of the LBVH key generation and ordering: 30-bit Morton codes
of triangle AABB centres and their stable order.  The device build
(ordinarylight_b200/csrc/olc_bvh.cu) must equal these bit for bit:

* centre = (min + max) * 0.5 per axis in float32;
* q = trunc(clip((c - lo) * (1 / (hi - lo)) * 1024, 0, 1023)) with lo/hi the
  centre bounds, every operation a single correctly rounded float32 step;
* code = interleave(qx, qy, qz) with x in the highest bit of each triple;
* order = numpy.argsort(codes, kind="stable") (equal codes keep input order).
"""

from __future__ import annotations

import numpy as np

__all__ = ["triangle_centers", "expand_bits10", "morton_codes", "stable_order"]


def triangle_centers(triangles):
    tri = np.asarray(triangles, np.float32).reshape(-1, 3, 3)
    lo = tri.min(axis=1)
    hi = tri.max(axis=1)
    return (lo + hi) * np.float32(0.5)


def expand_bits10(v):
    v = np.asarray(v, np.uint32)
    v = (v * np.uint32(0x00010001)) & np.uint32(0xFF0000FF)
    v = (v * np.uint32(0x00000101)) & np.uint32(0x0F00F00F)
    v = (v * np.uint32(0x00000011)) & np.uint32(0xC30C30C3)
    v = (v * np.uint32(0x00000005)) & np.uint32(0x49249249)
    return v


def morton_codes(triangles):
    c = triangle_centers(triangles)
    lo = c.min(axis=0)
    hi = c.max(axis=0)
    ext = (hi - lo).astype(np.float32)
    with np.errstate(divide="ignore"):
        inv = np.where(ext > 0, np.float32(1.0) / np.where(ext > 0, ext, np.float32(1.0)), np.float32(0.0))
    inv = inv.astype(np.float32)
    q = ((c - lo) * inv) * np.float32(1024.0)
    q = np.clip(q, np.float32(0.0), np.float32(1023.0)).astype(np.uint32)
    return (expand_bits10(q[:, 0]) << np.uint32(2)) | (expand_bits10(q[:, 1]) << np.uint32(1)) | expand_bits10(q[:, 2])


def stable_order(codes):
    return np.argsort(np.asarray(codes, np.uint32), kind="stable").astype(np.uint32)
