"""The denoiser on the device: guide pass + edge-avoiding A-Trous (gr_guide_buffers,
gr_atrous_denoise, gr_denoise_tonemap_device).

Mirrors crates/gemray/src/renderer/denoise/mod.rs (`AtrousParams`, `GBuffers`,
`AtrousDenoiser::denoise`), apps/diagram-gui/src/bridge/guide_pass.rs
(`generate_guide_buffers`) and apps/diagram-gui/src/bridge/render_thread/denoise.rs
(`denoise_and_tonemap_frame`) by name and argument meaning.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi
from .backend import GpuFrameRenderer, _raise_for
from .scene import Scene

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)


@dataclass
class AtrousParams:
    num_passes: int = 5
    sigma_color: float = 0.35
    sigma_depth: float = 0.1
    normal_power: float = 64.0
    taper_reference_spp: float = 4.0
    taper_identity_epsilon: float = 0.02

    def c(self) -> abi.gr_atrous_params:
        return abi.gr_atrous_params(self.num_passes, self.sigma_color, self.sigma_depth, self.normal_power,
                                    self.taper_reference_spp, self.taper_identity_epsilon)


@dataclass
class GuideBuffers:
    depth: np.ndarray     # (W*H,) f32, 1e6 on a miss
    normal: np.ndarray    # (W*H, 3) f32, zero on a miss
    facet_id: np.ndarray  # (W*H,) i32, -1 on a miss


def generate_guide_buffers(renderer: GpuFrameRenderer, scene: Scene) -> GuideBuffers:
    n = scene.width * scene.height
    g = GuideBuffers(np.empty(n, np.float32), np.empty((n, 3), np.float32), np.empty(n, np.int32))
    _raise_for(renderer.lib, renderer.lib.gr_guide_buffers(renderer.ctx, C.byref(scene.c_scene()),
                                                           g.depth.ctypes.data_as(_fp), g.normal.ctypes.data_as(_fp),
                                                           g.facet_id.ctypes.data_as(_ip)))
    return g


def denoise(renderer: GpuFrameRenderer, color: np.ndarray, guides: GuideBuffers, width: int, height: int, spp: int,
            params: AtrousParams | None = None) -> np.ndarray:
    """AtrousDenoiser::denoise on host buffers: the averaged XYZ image in, filtered out."""
    c = np.ascontiguousarray(color, np.float32).reshape(-1, 3)
    if c.shape[0] != width * height:
        raise ValueError("color must hold width * height pixels")
    out = np.empty_like(c)
    p = (params or AtrousParams()).c()
    _raise_for(renderer.lib, renderer.lib.gr_atrous_denoise(
        renderer.ctx, c.ctypes.data_as(_fp), np.ascontiguousarray(guides.depth, np.float32).ctypes.data_as(_fp),
        np.ascontiguousarray(guides.normal, np.float32).ctypes.data_as(_fp),
        np.ascontiguousarray(guides.facet_id, np.int32).ctypes.data_as(_ip), width, height, spp, C.byref(p),
        out.ctypes.data_as(_fp)))
    return out
