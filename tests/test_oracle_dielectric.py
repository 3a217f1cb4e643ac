"""Known answers for the dielectric oracle (CPU only): a slab at normal
incidence passes rays straight through with two interface factors; Snell's
law bends an oblique ray; total internal reflection turns a ray back."""

from __future__ import annotations

import numpy as np

from oracle import dielectric


def _slab(z0, z1, size=50.0):
    quads = []
    for z, flip in ((z0, False), (z1, True)):
        a, b, c, d = [(-size, -size, z), (size, -size, z), (size, size, z), (-size, size, z)]
        quads += [(a, b, c), (a, c, d)] if not flip else [(a, c, b), (a, d, c)]
    return np.array(quads, np.float64)


def test_slab_at_normal_incidence():
    tris = _slab(0.0, 1.0)
    env = np.full((4, 8, 3), 2.0, np.float32)
    o = np.array([[0.1, 0.2, -5.0]])
    d = np.array([[0.0, 0.0, 1.0]])
    n = len(tris)
    rad, robust = dielectric.trace(o, d, tris, np.full(n, 0.5), np.full(n, 1.5), np.tile([0.5, 1.0, 0.0], (n, 1)),
                                   env, texel_margin=0.0)
    factor = (0.8 + 0.2 * np.array([0.5, 1.0, 0.0])) * 0.5
    np.testing.assert_allclose(rad[0], 2.0 * factor ** 2, rtol=1e-6)


def test_snell_and_total_internal_reflection():
    ior = 1.5
    theta = np.radians(30.0)
    d = np.array([[np.sin(theta), 0.0, np.cos(theta)]])
    # one interface into glass: the direction inside obeys Snell's law
    w = dielectric._refract(d, np.array([[0.0, 0.0, -1.0]]), np.array([1.0 / ior]))
    w /= np.linalg.norm(w)
    assert np.isclose(np.sin(theta), ior * w[0, 0] / np.linalg.norm(w[0]), rtol=1e-9)
    # beyond the critical angle from inside: no transmitted direction
    steep = np.radians(50.0)
    d_in = np.array([[np.sin(steep), 0.0, np.cos(steep)]])
    assert not dielectric._refract(d_in, np.array([[0.0, 0.0, -1.0]]), np.array([ior])).any()
