"""The block-sorted kernel (GR_KERNEL_SORTED) against the plain kernel.

Every path runs the same functions in the same order, only the thread that advances it
changes, so films must be bit-identical to the plain kernel's: clear isotropic stones in
all three environment kinds, in one launch and split over several chunks (the tuple
counter restarts per launch), a 510-plane stone (the slot pool plus plane tables need
more than 48 KB of shared memory) and a max-depth-1 scene; scenes outside the class
(birefringent, absorbing, frosted) run AUTO's kernel and match as well."""
from __future__ import annotations

import numpy as np
import pytest

from gemray_studio_b200 import abi, scene as S, workloads as W
from helpers import srb_scene

pytestmark = pytest.mark.gpu


def film(sc, kernel, spp, offset=3, budget=0):
    from gemray_studio_b200 import GpuFrameRenderer
    r = GpuFrameRenderer(kernel=kernel, chunk_budget_bytes=budget)
    try:
        acc = np.zeros((sc.width * sc.height, 3), np.float32)
        r.accumulate(sc, offset, spp, acc)
        return acc
    finally:
        r.close()


def same(a, b):
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("env", [abi.GR_ENV_UNIFORM, abi.GR_ENV_STUDIO, abi.GR_ENV_LATLONG])
def test_sorted_matches_plain_clear_stones(engine_lib, env):
    sc = srb_scene("Diamond", width=64, height=48, max_bounces=32, env_mode=env,
                   latlong=S.gaussian_blob_latlong(256, 128, seed=1))
    ref = film(sc, abi.GR_KERNEL_PLAIN, 64)
    assert same(film(sc, abi.GR_KERNEL_SORTED, 64), ref)
    assert same(film(sc, abi.GR_KERNEL_SORTED, 64, budget=5000 * 12), ref)  # chunks of 78 pixels


def test_sorted_matches_plain_on_the_benchmark_stone(engine_lib):
    sc, _ = W.config_scene("c2s")
    sc.width, sc.height = 240, 136
    assert same(film(sc, abi.GR_KERNEL_SORTED, 16), film(sc, abi.GR_KERNEL_PLAIN, 16))


def test_sorted_many_planes_and_shallow(engine_lib):
    rng = np.random.default_rng(11)
    planes = S.random_polyhedron(rng, 500, 510)
    assert planes.shape[0] > 400
    sc = S.Scene(width=40, height=32, planes=planes, material=S.builtin_material("Cubic Zirconia"),
                 cam=S.camera(0.4, 0.3, 4.0, 30.0), max_bounces=24, env_mode=abi.GR_ENV_STUDIO)
    assert same(film(sc, abi.GR_KERNEL_SORTED, 32), film(sc, abi.GR_KERNEL_PLAIN, 32))
    sc1 = srb_scene("Diamond", width=32, height=32, max_bounces=1)
    assert same(film(sc1, abi.GR_KERNEL_SORTED, 8), film(sc1, abi.GR_KERNEL_PLAIN, 8))


@pytest.mark.parametrize("material", ["Sapphire", "Tourmaline"])
def test_sorted_mode_outside_its_class_runs_auto(engine_lib, material):
    sc = srb_scene(material, width=40, height=30, max_bounces=24)
    assert same(film(sc, abi.GR_KERNEL_SORTED, 32), film(sc, abi.GR_KERNEL_PLAIN, 32))
    sc.finishes = np.zeros(sc.planes.shape[0], np.uint32)
    sc.finishes[3] = 1
    sc.material = S.builtin_material("Diamond")
    assert same(film(sc, abi.GR_KERNEL_SORTED, 16), film(sc, abi.GR_KERNEL_PLAIN, 16))
