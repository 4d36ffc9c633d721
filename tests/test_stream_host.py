"""Host-side pieces of the frame-delta streaming path that need no GPU: the radiance
wire codec (crates/gemray-net/src/radiance/mod.rs:26-67 and its tests), the
sub-batch sizing rule as the library implements it (stream_emit/sizing.rs:22-30 and
tests.rs:75-92), and the oracle's downsample_preview (downsample.rs:17-53,
tests.rs:94-107)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gemray_studio_b200 import radiance


def test_bytes_per_pixel_is_three_f32():
    assert radiance.BYTES_PER_PIXEL == 12


def test_radiance_round_trips_bit_exactly():
    film = np.array([[1.0, 2.0, 3.0], [-0.5, np.finfo(np.float32).max, 0.0], [0.0, 0.0, 0.0]], np.float32)
    b = radiance.encode(film)
    assert len(b) == 36
    back = radiance.decode(b, 3, 1)
    assert back.tobytes() == film.tobytes()
    assert b[:4] == np.float32(1.0).tobytes()  # little-endian f32, pixel-major


@pytest.mark.parametrize("mutate", ["short", "long", "empty"])
def test_radiance_rejects_wrong_lengths(mutate):
    b = radiance.encode(np.ones((4, 3), np.float32))
    bad = {"short": b[:-1], "long": b + b"\0", "empty": b""}[mutate]
    with pytest.raises(radiance.RadianceError):
        radiance.decode(bad, 2, 2)


def test_radiance_empty_frame():
    assert radiance.decode(b"", 0, 5).shape == (0, 3)


def _reference_next_batch_size(prev: int, elapsed_ms: float, target_ms: float = 100.0) -> int:
    max_growth = max(min(prev * 4, 0xFFFFFFFF), 1)
    if elapsed_ms == 0:
        return max_growth
    scaled = prev * (target_ms / elapsed_ms)
    v = min(max(scaled, 1.0), float(max_growth))
    return int(np.floor(v + 0.5))  # f64::round: half away from zero (v >= 1)


def test_next_batch_size_rule(engine_lib):
    f = engine_lib.gr_next_batch_size
    assert f(4, 10.0, 100.0) > 4
    n = f(100, 400.0, 100.0)
    assert 1 <= n < 100
    assert f(0, 1.0, 100.0) >= 1 and f(1, 10000.0, 100.0) >= 1
    assert f(7, 0.0, 100.0) == 28 and f(0, 0.0, 100.0) == 1
    assert f(0xFFFFFFFF, 0.0, 100.0) == 0xFFFFFFFF  # saturating growth
    rng = np.random.default_rng(3)
    for prev in [1, 2, 3, 17, 250, 4096, 1 << 20]:
        for ms in np.concatenate([rng.uniform(0.01, 1000.0, 20), [25.0, 50.0, 100.0, 400.0]]):
            assert f(prev, float(ms), 100.0) == _reference_next_batch_size(prev, float(ms)), (prev, ms)


def _preview(oracle, src: np.ndarray, w: int, h: int, tw: int, th: int) -> np.ndarray:
    out = np.empty((max(tw, 1) * max(th, 1), 3), np.float32)
    fp = C.POINTER(C.c_float)
    oracle.gro_downsample_preview(np.ascontiguousarray(src, np.float32).ctypes.data_as(fp), w, h, tw, th,
                                  out.ctypes.data_as(fp))
    return out


def test_downsample_preview_dimensions_and_uniform_value(oracle):
    assert _preview(oracle, np.ones((64, 3), np.float32), 8, 8, 2, 2).shape == (4, 3)
    uni = np.tile(np.array([2.0, 4.0, 6.0], np.float32), (64, 1))
    out = _preview(oracle, uni, 8, 8, 2, 2)
    assert np.all(np.abs(out - np.array([2.0, 4.0, 6.0])) < 1e-5)


def test_downsample_preview_is_the_block_mean(oracle):
    rng = np.random.default_rng(0)
    w, h = 13, 7
    src = rng.uniform(0, 5, (w * h, 3)).astype(np.float32)
    for tw, th in [(5, 3), (13, 7), (20, 11), (1, 1), (0, 0)]:
        out = _preview(oracle, src, w, h, tw, th)
        TW, TH = max(tw, 1), max(th, 1)
        img = src.reshape(h, w, 3).astype(np.float64)
        for oy in range(TH):
            y0 = oy * h // TH
            y1 = min(max((oy + 1) * h // TH, y0 + 1), h)
            for ox in range(TW):
                x0 = ox * w // TW
                x1 = min(max((ox + 1) * w // TW, x0 + 1), w)
                ref = img[y0:y1, x0:x1].reshape(-1, 3).mean(axis=0)
                assert np.allclose(out[oy * TW + ox], ref, rtol=1e-6), (tw, th, ox, oy)
