"""Synthetic inputs of the reference's denoiser tests (crates/gemray/src/renderer/
denoise/mod.rs tests, crates/gemray/tests/denoise_tests.rs): the Xorshift32 stream and
the irregular guide-buffer scene, restated."""
from __future__ import annotations

import numpy as np


class Xorshift32:
    def __init__(self, seed: int):
        self.s = seed if seed != 0 else 0xDEADBEEF

    def next_u32(self) -> int:
        x = self.s
        x ^= (x << 13) & 0xFFFFFFFF
        x ^= x >> 17
        x ^= (x << 5) & 0xFFFFFFFF
        self.s = x
        return x

    def next_f32(self) -> np.float32:
        return np.float32(float(self.next_u32()) / float(0xFFFFFFFF))

    def next_signed(self) -> np.float32:
        # f32 mul_add(2, -1): exact in f64, then one rounding
        return np.float32(np.float64(self.next_f32()) * 2.0 - 1.0)


def unit(v) -> np.ndarray:
    v = np.asarray(v, np.float32)
    return v * (np.float32(1.0) / np.float32(np.sqrt(np.float32((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]))))


def irregular_scene(width: int, height: int, seed: int):
    """color, depth, normal, facet_id of the reference's `irregular_scene`."""
    rng = Xorshift32(seed)
    n = width * height
    color = np.zeros((n, 3), np.float32)
    depth = np.zeros(n, np.float32)
    normal = np.zeros((n, 3), np.float32)
    facet = np.zeros(n, np.int32)
    for y in range(height):
        for x in range(width):
            i = y * width + x
            facet[i] = (x // 5 + y // 7) % 6
            depth[i] = rng.next_f32() * np.float32(4.0)
            jx = rng.next_signed() * np.float32(0.3)
            jy = rng.next_signed() * np.float32(0.3)
            normal[i] = unit([jx, jy, 1.0])
            color[i] = [rng.next_f32(), rng.next_f32(), rng.next_f32()]
    return color, depth, normal, facet
