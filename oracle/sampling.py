"""ORACLE — test infrastructure only, never part of the product path.

Host restatement of the renderer's counter-based sampling sequence and
camera model, used to check the device raygen:

* hash(v): xor-shift 16, * 0x7feb352d, xor-shift 15, * 0x846ca68b,
  xor-shift 16 (the reference wavefront's waveHash,
  ordinarylight/shaders/wavefront_generate.comp:71-79);
* seed(pixel, sample, frame) = hash(hash(pixel ^ hash(frame)) ^ hash(sample + 1))
  (the reference's wavefront_generate.comp:113-116 mixes the same three
  hashes with one xor, which makes frame f / sample s collide with
  frame s + 1 / sample f - 1; the pixel/frame hash is nested first here);
* camera jitter = two further hash steps of the seed, each / 2^32
  (wavefront_generate.comp:117-121);
* per-bounce stream: hash(seed ^ hash(bounce * 0x9e3779b9 + 0x632be5ab)),
  then PCG-RXS-M-XS draws (randomFloat, transport_v1/sampling.glsl:16-22).
"""

from __future__ import annotations

import numpy as np

__all__ = ["hash32", "path_seed", "camera_jitter", "bounce_state", "pcg_draws"]

_M32 = 0xFFFFFFFF


def hash32(v):
    v = np.asarray(v, np.uint64) & _M32
    v ^= v >> 16
    v = (v * 0x7FEB352D) & _M32
    v ^= v >> 15
    v = (v * 0x846CA68B) & _M32
    v ^= v >> 16
    return v.astype(np.uint32)


def path_seed(pixel, sample, frame):
    pixel = np.asarray(pixel, np.uint32)
    inner = hash32(pixel ^ hash32(np.uint32(frame))) ^ hash32((np.asarray(sample, np.uint64) + 1) & _M32)
    return hash32(inner)


def camera_jitter(pixel, sample, frame):
    s = hash32(path_seed(pixel, sample, frame))
    jx = s.astype(np.float32) * np.float32(1.0 / 4294967296.0)
    s = hash32(s)
    jy = s.astype(np.float32) * np.float32(1.0 / 4294967296.0)
    return jx, jy


def bounce_state(seed, bounce):
    key = (np.asarray(bounce, np.uint64) * 0x9E3779B9 + 0x632BE5AB) & _M32
    return hash32(np.asarray(seed, np.uint32) ^ hash32(key))


def pcg_draws(state, count):
    """``count`` PCG-RXS-M-XS draws from each state; returns (draws, state)."""
    s = np.asarray(state, np.uint64) & _M32
    out = []
    for _ in range(count):
        s = (s * 747796405 + 2891336453) & _M32
        word = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & _M32
        word = (word >> 22) ^ word
        out.append(word.astype(np.uint32).astype(np.float32) * np.float32(1.0 / 4294967296.0))
    return np.stack(out, axis=-1), s.astype(np.uint32)
