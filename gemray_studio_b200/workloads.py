"""Seeded synthetic workloads for the batched (many stones per launch) and served
(request stream) forms of the transport path.

* `material_tables()` -- six materials spanning n_d 1.46 to 2.42: a Cauchy crown
  glass with two absorption bands, quartz, spinel, sapphire, zircon and diamond (the
  last five are the reference's built-in materials, optics/materials.rs).
* `random_stones(n, ...)` -- n scenes, each a random convex polyhedron of 17-145
  facet planes (normals by rejection-sampled sphere points, offsets U[0.8, 1.0],
  symmetrised by a random 4-16-fold rotation about +Y), a material drawn from the
  tables, square films and spp drawn log-uniformly from the given ranges, Kahan film
  sums, a seeded lat-long environment.
* `request_stream(...)` -- Poisson arrivals of render requests over such stones, with
  a share of metric-only pose sweeps.

There is no dataset for this path in the reference; every input is generated here
from the seed.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi
from . import scene as S


def _crown_glass() -> abi.gr_material:
    """Cauchy crown glass, n = 1.4580 + 0.00354 / lambda^2 (lambda in um, n_d = 1.4682),
    isotropic, two weak Gaussian absorption bands (a faint blue-green tint)."""
    m = S.builtin_material("Spinel")  # isotropic template; every optical field is overwritten
    d = m.dispersion
    d.model_type = abi.GR_DISP_CAUCHY
    d.param_a[0], d.param_a[1], d.param_a[2], d.param_a[3] = 1.4580, 0.00354, 0.0, 0.0
    for i in range(4):
        d.param_b[i] = 0.0
        d.param_c[i] = 0.0
    m.o_ray_band_count = 2
    m.e_ray_band_count = 2
    bands = [(620.0, 45.0, 0.35), (430.0, 30.0, 0.2)]
    for k, (c, w, p) in enumerate(bands):
        m.o_ray_bands[k].center_nm, m.o_ray_bands[k].width_nm, m.o_ray_bands[k].peak = c, w, p
        m.e_ray_bands[k].center_nm, m.e_ray_bands[k].width_nm, m.e_ray_bands[k].peak = c, w, p
    return m


_KEEP: list = []  # tables the extension structs point at


def birefringent_emerald_material(lambda_dependent: bool = True, seed: int = 0,
                                  path_scale: float = 0.1) -> tuple[abi.gr_material, abi.gr_material_ext]:
    """The step-cut emerald's uniaxial, dichroic material: Cauchy indices
    n_o = 1.640 + 0.0042 / lambda^2 and n_e = 1.620 + 0.0040 / lambda^2 (lambda in um);
    with `lambda_dependent` the extraordinary index follows its own Cauchy law (the
    material extension), otherwise Delta n = n_e - n_o at 589.3 nm is constant; c-axis
    uniform on the sphere from `seed`; absorption (cm^-1) o: 0.8 / 0.3 / 0.1 and
    e: 0.2 / 0.6 / 1.2 at 450 / 550 / 650 nm, linearly interpolated (held flat outside)
    and tabulated at 5 nm from 380 to 780 nm; `path_scale` converts model units to cm
    (0.1: one model unit is 1 mm)."""
    lam = 0.5893
    n_o = 1.640 + 0.0042 / lam ** 2
    n_e = 1.620 + 0.0040 / lam ** 2
    m = S.custom_material(1.640 + 0.0042 / lam ** 2, 0.0, n_e - n_o)
    d = m.dispersion
    d.model_type = abi.GR_DISP_CAUCHY
    d.param_a[0], d.param_a[1], d.param_a[2], d.param_a[3] = 1.640, 0.0042, 0.0, 0.0
    rng = np.random.default_rng(seed)
    while True:
        c = rng.uniform(-1.0, 1.0, 3)
        r2 = float(c @ c)
        if 1e-6 < r2 <= 1.0:
            break
    c = (c / math.sqrt(r2)).astype(np.float32)
    d.c_axis_and_birefringence[0], d.c_axis_and_birefringence[1], d.c_axis_and_birefringence[2] = (float(x) for x in c)
    grid = np.arange(380.0, 780.0 + 1e-3, 5.0)
    knots = np.array([450.0, 550.0, 650.0])
    a_o = np.interp(grid, knots, [0.8, 0.3, 0.1]).astype(np.float32)
    a_e = np.interp(grid, knots, [0.2, 0.6, 1.2]).astype(np.float32)
    ext = abi.gr_material_ext()
    ext.n_absorption = len(grid)
    ext.absorption_nm_first = 380.0
    ext.absorption_nm_step = 5.0
    ext.alpha_o_table = a_o.ctypes.data_as(C.POINTER(C.c_float))
    ext.alpha_e_table = a_e.ctypes.data_as(C.POINTER(C.c_float))
    ext.has_cauchy_e = 1 if lambda_dependent else 0
    ext.cauchy_e[0], ext.cauchy_e[1], ext.cauchy_e[2] = 1.620, 0.0040, 0.0
    _KEEP.append((a_o, a_e))
    m.absorption_path_scale = path_scale
    return m, ext


# The single-scene benchmark configurations: c1 (CPU-runnable), c2 (the headline
# frame), c3 (the birefringent dichroic emerald) and c2s (c2's scene at 480x270, 64 spp,
# the small case of the profiler captures).
CONFIGS = {
    "c1": dict(width=256, height=256, spp=64, max_bounces=32, env="uniform", stone="rb57"),
    "c2": dict(width=1920, height=1080, spp=256, max_bounces=32, env="latlong", stone="rb57"),
    "c3": dict(width=1024, height=1024, spp=1024, max_bounces=64, env="studio", stone="em49"),
    "c2s": dict(width=480, height=270, spp=64, max_bounces=32, env="latlong", stone="rb57"),
}


def config_scene(name: str, camera=None, builtin_material=None, lambda_dependent: bool = True):
    """The scene of benchmark configuration `name` and its sizes (CONFIGS[name]).

    c1/c2: the 57-facet round brilliant (table 57%, crown 34.5 deg, pavilion 40.75 deg,
    16 girdle planes), Diamond, camera Camera::new(0.35, 0.28, 5.0, 18.0); c1 in a
    uniform white environment, c2 in the seeded 2048x1024 lat-long map of 12 Gaussian
    lights.  c3: the 49-plane step-cut emerald with birefringent_emerald_material()
    (lambda_dependent=False: the reference model's constant Delta n) in the studio rig.
    `camera` / `builtin_material` replace the scene builders (Camera::new and the
    built-in material table) -- the engine library's by default."""
    camera = camera or S.camera
    builtin_material = builtin_material or S.builtin_material
    w = CONFIGS[name]
    planes = S.round_brilliant_57() if w["stone"] == "rb57" else S.emerald_cut_49()
    env_mode = {"uniform": abi.GR_ENV_UNIFORM, "latlong": abi.GR_ENV_LATLONG, "studio": abi.GR_ENV_STUDIO}[w["env"]]
    latlong = S.gaussian_blob_latlong(2048, 1024, 12, seed=0) if w["env"] == "latlong" else None
    ext = None
    if w["stone"] == "rb57":
        mat = builtin_material("Diamond")
    else:
        mat, ext = birefringent_emerald_material(lambda_dependent=lambda_dependent)
    sc = S.Scene(width=w["width"], height=w["height"], planes=planes, material=mat, cam=camera(0.35, 0.28, 5.0, 18.0),
                 max_bounces=w["max_bounces"], env_mode=env_mode, latlong=latlong, uniform_rgb=(1.0, 1.0, 1.0),
                 ext=ext)
    return sc, dict(w)


def material_tables() -> list[tuple[str, abi.gr_material]]:
    return [("crown glass", _crown_glass())] + [(n, S.builtin_material(n)) for n in
                                                ("Quartz", "Spinel", "Sapphire", "Zircon", "Diamond")]


@dataclass
class Stone:
    scene: S.Scene
    spp: int
    material: str
    n_planes: int


def _log_uniform_int(rng, lo: int, hi: int) -> int:
    return int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))


def random_stones(n: int = 64, seed: int = 0, side=(128, 1024), spp=(32, 512), max_bounces: int = 32,
                  env_size=(1024, 512)) -> list[Stone]:
    rng = np.random.default_rng(seed)
    mats = material_tables()
    env = S.gaussian_blob_latlong(env_size[0], env_size[1], 12, seed=seed)
    out = []
    for _ in range(n):
        planes = S.random_polyhedron(rng)
        name, mat = mats[int(rng.integers(0, len(mats)))]
        s = _log_uniform_int(rng, side[0], side[1])
        cam = S.camera(float(rng.uniform(-math.pi, math.pi)), float(rng.uniform(0.15, 0.9)), 4.0, 30.0)
        sc = S.Scene(width=s, height=s, planes=planes, material=mat, cam=cam, max_bounces=max_bounces,
                     env_mode=abi.GR_ENV_LATLONG, latlong=env, flags=abi.GR_FLAG_KAHAN_FILM)
        out.append(Stone(sc, _log_uniform_int(rng, spp[0], spp[1]), name, planes.shape[0]))
    return out


@dataclass
class Request:
    arrival_s: float
    stone: int                      # index into the stones list
    spp: int = 0                    # render
    poses: np.ndarray | None = None  # metrics-only sweep (n, 4): cam_yaw, cam_pitch, light_yaw, light_pitch
    extra: dict = field(default_factory=dict)

    @property
    def is_metrics(self) -> bool:
        return self.poses is not None


def request_stream(stones: list[Stone], rate_hz: float, duration_s: float, seed: int = 1, metrics_share: float = 0.1,
                   spp=(16, 1024), n_tilts: int = 64) -> list[Request]:
    """Poisson arrivals at rate_hz for duration_s; each request renders a random stone
    with log-uniform spp, or (metrics_share of them) sweeps n_tilts tilts in
    [-20, +20] deg around pitch 0.45 for that stone."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / rate_hz))
        if t > duration_s:
            break
        k = int(rng.integers(0, len(stones)))
        if rng.uniform() < metrics_share:
            tilts = np.deg2rad(np.linspace(-20.0, 20.0, n_tilts)).astype(np.float32)
            poses = np.stack([np.zeros(n_tilts, np.float32), np.float32(0.45) + tilts,
                              np.full(n_tilts, 0.85, np.float32), np.full(n_tilts, 0.95, np.float32)], axis=1)
            out.append(Request(t, k, poses=poses))
        else:
            out.append(Request(t, k, spp=_log_uniform_int(rng, spp[0], spp[1])))
    return out


def c2_tilt_poses(n: int = 16) -> np.ndarray:
    """The C2 metric sweep: n tilts uniformly in [-20, +20] deg around pitch 0.45,
    camera yaw 0, light (0.85, 0.95)."""
    tilts = np.deg2rad(np.linspace(-20.0, 20.0, n)).astype(np.float32)
    return np.stack([np.zeros(n, np.float32), np.float32(0.45) + tilts, np.full(n, 0.85, np.float32),
                     np.full(n, 0.95, np.float32)], axis=1)
