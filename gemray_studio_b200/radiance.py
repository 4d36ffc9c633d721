"""The radiance wire codec (crates/gemray-net/src/radiance/mod.rs:26-67): a film of
per-pixel running XYZ sums travels as its raw little-endian f32 bytes, 12 per pixel,
in pixel order -- the layout the engine's films already have, so encoding is a byte
view and decoding a length-checked copy.
"""
from __future__ import annotations

import numpy as np

BYTES_PER_PIXEL = 12  # size_of::<Vec3>()


class RadianceError(ValueError):
    """A FRAME payload whose length is not width * height * BYTES_PER_PIXEL
    (RadianceError::LengthMismatch).  Python buffers are copied on decode, so the
    reference's Misaligned case cannot arise here."""

    def __init__(self, width: int, height: int, expected_bytes: int, got_bytes: int):
        super().__init__(f"radiance payload for {width}x{height} must be {expected_bytes} bytes, got {got_bytes}")
        self.width, self.height = width, height
        self.expected_bytes, self.got_bytes = expected_bytes, got_bytes


def encode(film: np.ndarray) -> bytes:
    """radiance::encode: the film's (N, 3) float32 values as little-endian bytes."""
    f = np.asarray(film)
    if f.dtype != np.float32 or f.ndim != 2 or f.shape[1] != 3:
        raise ValueError("a radiance buffer is an (N, 3) float32 array")
    return np.ascontiguousarray(f, dtype="<f4").tobytes()


def decode(payload: bytes | bytearray | memoryview, width: int, height: int) -> np.ndarray:
    """radiance::decode: validate the length against width * height, then return a
    (width * height, 3) float32 copy.  An empty frame decodes to an empty array."""
    expected = int(width) * int(height) * BYTES_PER_PIXEL
    got = len(payload)
    if got != expected:
        raise RadianceError(width, height, expected, got)
    if expected == 0:
        return np.zeros((0, 3), np.float32)
    return np.frombuffer(bytes(payload), dtype="<f4").astype(np.float32).reshape(-1, 3)
