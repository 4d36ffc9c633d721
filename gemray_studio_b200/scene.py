"""Scene description for the engine: facet planes + material + camera + environment.

`Scene` mirrors the reference's ``GpuSceneRef`` (crates/gemray/src/renderer/gpu_backend.rs:85-99)
and owns every array a ``gr_scene`` borrows.  The helpers build:

* the reference's own inputs through the engine library (bit-identical f32 libm
  arithmetic): ``camera`` = ``Camera::new`` (optics/raytracer/camera.rs:62-93),
  ``standard_round_brilliant`` (geometry/cuts.rs:45-129), ``builtin_material``
  (optics/materials.rs:136-1250 encoded as renderer/buffers.rs GpuGemMaterial);
* seeded synthetic inputs with the shapes of the benchmark workloads (a 57-facet
  round brilliant with table 57% / crown 34.5 deg / pavilion 40.75 deg, a 49-facet
  step-cut emerald, random symmetric convex polyhedra, a lat-long environment of
  Gaussian light blobs).  These have no counterpart in the reference.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi

# LightingPreset::params() (optics/raytracer/environment.rs:81-100): (temp_k, spot_mult)
LIGHTING_PRESETS = {
    "Daylight": (6500.0, 1.0),
    "Incandescent": (3200.0, 1.2),
    "RingLights": (5000.0, 1.6),
    "DarkSpotlight": (6000.0, 2.4),
}

BUILTIN_MATERIALS = (
    "Diamond", "Sapphire", "Ruby", "Emerald", "Zircon", "Alexandrite", "Topaz", "Spinel", "Quartz",
    "Tourmaline", "Tanzanite", "Synthetic Moissanite", "Cubic Zirconia",
)


def _lib():
    return abi.load_library()


def camera(yaw: float, pitch: float, distance: float, fov_deg: float) -> abi.gr_camera:
    cam = abi.gr_camera()
    st = _lib().gr_camera_new(yaw, pitch, distance, fov_deg, C.byref(cam))
    assert st == abi.GR_OK
    return cam


def standard_round_brilliant() -> np.ndarray:
    """The reference's 74-plane standard round brilliant, (74, 4) float32 [nx, ny, nz, d]."""
    buf = (abi.gr_plane * 128)()
    n = _lib().gr_standard_round_brilliant(buf, 128)
    return np.ctypeslib.as_array(buf).view(np.float32).reshape(-1, 4)[:n].copy()


def custom_material(mean_ri: float, dispersion_delta: float, birefringence_delta: float,
                    absorption_rgb=(0.0, 0.0, 0.0)) -> abi.gr_material:
    """= GpuGemMaterial::encode(&GemMaterial::new_custom(..)) (optics/materials.rs:1257-1316,
    renderer/buffers.rs:655-800): a Cauchy fit through n_d with the given F-C
    dispersion (f32 arithmetic as the reference), c-axis +Y, trigonal / uniaxial when
    |birefringence| > 1e-4, absorption as legacy_rgb_bands (optics/absorption.rs:179-185)
    on both eigenmodes."""
    f = np.float32
    ld, lf, lc = f(0.5893), f(0.4861), f(0.6563)
    k_fc = f(1.0) / (f(1.0) / (lf * lf) - f(1.0) / (lc * lc))
    b = max(f(dispersion_delta) * k_fc, f(0.0))
    a = max(f(mean_ri) - b / (ld * ld), f(1.0))
    bire = f(birefringence_delta)
    m = abi.gr_material()
    d = m.dispersion
    d.model_type = abi.GR_DISP_CAUCHY
    d.param_a[0], d.param_a[1] = float(a), float(b)
    d.c_axis_and_birefringence[1] = 1.0
    d.c_axis_and_birefringence[3] = float(bire)
    aniso = abs(float(bire)) > 1e-4
    d.is_anisotropic = 1 if aniso else 0
    m.crystal_system = 3 if aniso else 0  # Trigonal / Cubic
    m.optical_character = 1 if bire > 1e-4 else (2 if bire < -1e-4 else 0)
    for k, (c, w, p) in enumerate(((620.0, 55.0, absorption_rgb[0]), (540.0, 45.0, absorption_rgb[1]),
                                    (450.0, 45.0, absorption_rgb[2]))):
        for bands in (m.o_ray_bands, m.e_ray_bands):
            bands[k].center_nm, bands[k].width_nm, bands[k].peak = c, w, p
    for first, bands in ((3, m.o_ray_bands), (3, m.e_ray_bands), (0, m.beta_ray_bands)):  # unused slots: width 1
        for k in range(first, abi.GR_MAX_BANDS):
            bands[k].width_nm = 1.0
    m.o_ray_band_count = m.e_ray_band_count = 3
    m.absorption_path_scale = 1.0
    return m


def builtin_material(name: str) -> abi.gr_material:
    m = abi.gr_material()
    st = _lib().gr_builtin_material(name.encode(), C.byref(m))
    if st != abi.GR_OK:
        raise KeyError(name)
    return m


def plane_from_normal(n, d: float) -> list[float]:
    """GpuFacetPlane::new: normalise in f32 with glam's v * (1/len)."""
    v = np.asarray(n, dtype=np.float32)
    dd = np.float32(np.float32(v[0] * v[0]) + np.float32(v[1] * v[1])) + np.float32(v[2] * v[2])
    r = np.float32(1.0) / np.sqrt(np.float32(dd))
    u = (v * r).astype(np.float32)
    return [float(u[0]), float(u[1]), float(u[2]), float(np.float32(d))]


def _crown_plane(theta_deg: float, az: float, r: float, y: float, sign: float = 1.0) -> list[float]:
    """Plane tilted theta_deg from the girdle plane, facing azimuth az, through the
    point at horizontal radius r (along az) and height y; sign -1 for the pavilion."""
    t = math.radians(theta_deg)
    n = [math.sin(t) * math.cos(az), sign * math.cos(t), math.sin(t) * math.sin(az)]
    d = -(n[0] * r * math.cos(az) + n[1] * y + n[2] * r * math.sin(az))
    return plane_from_normal(n, d)


def round_brilliant_57(table_pct: float = 57.0, crown_deg: float = 34.5, pavilion_deg: float = 40.75,
                       girdle_half: float = 0.015) -> np.ndarray:
    """57-facet round brilliant -- table, 8 stars, 8 bezels (crown mains), 16 upper
    halves, 16 lower halves, 8 pavilion mains; pointed culet -- plus the 16 vertical
    girdle planes of the reference construction (geometry/cuts.rs:45-129): 73 planes,
    girdle radius 1, table diameter table_pct % of the girdle diameter, bezels at
    crown_deg, pavilion mains at pavilion_deg.  Star / half tilts keep the reference
    SRB's ratios (15:34.5, 41:34.5, 42.5:41)."""
    g = girdle_half
    table_r = table_pct / 100.0
    table_y = g + (1.0 - table_r) * math.tan(math.radians(crown_deg))
    planes = [plane_from_normal([0.0, 1.0, 0.0], -table_y)]
    step = 2.0 * math.pi / 96.0
    star_deg = crown_deg * 15.0 / 34.5
    for gi in [6, 18, 30, 42, 54, 66, 78, 90]:
        planes.append(_crown_plane(star_deg, gi * step, table_r * 0.93, table_y))
    for gi in [0, 12, 24, 36, 48, 60, 72, 84]:
        planes.append(_crown_plane(crown_deg, gi * step, 1.0, g))
    upper_deg = crown_deg * 41.0 / 34.5
    for gi in [95, 1, 11, 13, 23, 25, 35, 37, 47, 49, 59, 61, 71, 73, 83, 85]:
        planes.append(_crown_plane(upper_deg, gi * step, 1.0, g))
    for i in range(16):
        phi = 2.0 * math.pi * i / 16.0
        planes.append(plane_from_normal([math.cos(phi), 0.0, math.sin(phi)], -1.0))
    for gi in [0, 12, 24, 36, 48, 60, 72, 84]:
        planes.append(_crown_plane(pavilion_deg, gi * step, 1.0, -g, -1.0))
    lower_deg = pavilion_deg * 42.5 / 41.0
    for gi in [95, 1, 11, 13, 23, 25, 35, 37, 47, 49, 59, 61, 71, 73, 83, 85]:
        planes.append(_crown_plane(lower_deg, gi * step, 1.0, -g, -1.0))
    return np.asarray(planes, np.float32)


def emerald_cut_49(length_width: float = 1.5, girdle_half: float = 0.015) -> np.ndarray:
    """49-plane step-cut emerald: table + 3 crown steps x 8 (4 sides + 4 cut corners)
    + 8 girdle planes + 4 pavilion steps x 4 sides, girdle outline length:width =
    length_width (long axis x)."""
    g = girdle_half
    hz = 0.8
    hx = hz * length_width
    corner = 0.86 * (hx + hz) / math.sqrt(2.0)
    dirs = [(0.0, hx), (math.pi / 2, hz), (math.pi, hx), (3 * math.pi / 2, hz),
            (math.pi / 4, corner), (3 * math.pi / 4, corner), (5 * math.pi / 4, corner), (7 * math.pi / 4, corner)]
    crown_angles = [44.0, 36.0, 26.0]
    crown_y = [g, g + 0.10, g + 0.19, g + 0.26]  # crease heights; the last is the table
    planes = [plane_from_normal([0.0, 1.0, 0.0], -crown_y[-1])]
    for k, ang in enumerate(crown_angles):
        for az, r0 in dirs:
            r = r0
            for j in range(k):
                r -= (crown_y[j + 1] - crown_y[j]) / math.tan(math.radians(crown_angles[j]))
            planes.append(_crown_plane(ang, az, r, crown_y[k]))
    for az, r0 in dirs:
        planes.append(plane_from_normal([math.cos(az), 0.0, math.sin(az)], -r0))
    pav_angles = [58.0, 50.0, 42.0, 34.0]
    pav_y = [g, g + 0.22, g + 0.40, g + 0.53]
    for k, ang in enumerate(pav_angles):
        for az, r0 in dirs[:4]:
            r = r0
            for j in range(k):
                r -= (pav_y[j + 1] - pav_y[j]) / math.tan(math.radians(pav_angles[j]))
            planes.append(_crown_plane(ang, az, r, -pav_y[k], -1.0))
    return np.asarray(planes, np.float32)


def face_count(planes: np.ndarray) -> int:
    """Number of planes that bound a face of positive area of the convex solid."""
    from scipy.spatial import HalfspaceIntersection, ConvexHull
    hs = np.concatenate([planes[:, :3].astype(np.float64), planes[:, 3:4].astype(np.float64)], axis=1)
    pts = HalfspaceIntersection(hs, np.zeros(3)).intersections
    hull = ConvexHull(pts)
    used = set()
    for eq in hull.equations:
        n, d = eq[:3], eq[3]
        dots = planes[:, :3] @ n
        k = int(np.argmax(dots - 10 * np.abs(planes[:, 3] - d)))
        used.add(k)
    return len(used)


def random_polyhedron(rng: np.random.Generator, n_min: int = 17, n_max: int = 145) -> np.ndarray:
    """Random convex polyhedron: normals by rejection-sampled sphere points, offsets
    U[0.8, 1.0], made symmetric under a random 4-16-fold rotation about +Y."""
    fold = int(rng.integers(4, 17))
    n_target = int(rng.integers(n_min, n_max + 1))
    base = max(1, n_target // fold)
    planes: list[list[float]] = []
    while len(planes) < base * fold:
        p = rng.uniform(-1.0, 1.0, 3)
        r2 = float(p @ p)
        if r2 > 1.0 or r2 < 1e-4:
            continue
        p = p / math.sqrt(r2)
        d = float(rng.uniform(0.8, 1.0))
        for k in range(fold):
            a = 2.0 * math.pi * k / fold
            ca, sa = math.cos(a), math.sin(a)
            n = [ca * p[0] + sa * p[2], p[1], -sa * p[0] + ca * p[2]]
            planes.append(plane_from_normal(n, -d))
    # cap top and bottom so the solid is bounded even for unlucky draws
    planes.append(plane_from_normal([0.0, 1.0, 0.0], -0.9))
    planes.append(plane_from_normal([0.0, -1.0, 0.0], -0.9))
    arr = np.asarray(planes[: max(n_min, min(n_max, len(planes)))], np.float32)
    return arr


def gaussian_blob_latlong(w: int = 2048, h: int = 1024, n_blobs: int = 12, seed: int = 0) -> np.ndarray:
    """Black lat-long map plus n_blobs Gaussian lights: centres uniform on the upper
    hemisphere, sigma U[2, 6] deg, radiance log-uniform in [1, 100] (grey), all from
    `seed`.  Returns (h, w, 3) float32, row 0 at the +Y pole (env_map.rs:231-239)."""
    rng = np.random.default_rng(seed)
    v = (np.arange(h, dtype=np.float64) + 0.5) / h
    u = (np.arange(w, dtype=np.float64) + 0.5) / w
    theta = v * math.pi
    phi = u * 2.0 * math.pi
    st, ct = np.sin(theta)[:, None], np.cos(theta)[:, None]
    dirs = np.stack([st * np.sin(phi)[None, :], np.broadcast_to(ct, (h, w)), st * np.cos(phi)[None, :]], -1)
    img = np.zeros((h, w, 3), np.float64)
    for _ in range(n_blobs):
        z = rng.uniform(0.0, 1.0)           # cos(theta) uniform on the upper hemisphere
        az = rng.uniform(0.0, 2.0 * math.pi)
        s = math.sqrt(max(0.0, 1.0 - z * z))
        c = np.array([s * math.sin(az), z, s * math.cos(az)])
        sigma = math.radians(rng.uniform(2.0, 6.0))
        L = math.exp(rng.uniform(math.log(1.0), math.log(100.0)))
        ang = np.arccos(np.clip(dirs @ c, -1.0, 1.0))
        img += (L * np.exp(-0.5 * (ang / sigma) ** 2))[..., None]
    return img.astype(np.float32)


@dataclass
class Scene:
    """One render scene; keeps every borrowed array alive for the C call."""

    width: int
    height: int
    planes: np.ndarray
    material: abi.gr_material
    cam: abi.gr_camera
    max_bounces: int = 32
    env_mode: int = abi.GR_ENV_STUDIO
    uniform_rgb: tuple = (1.0, 1.0, 1.0)
    preset: str = "RingLights"
    exposure: float = 1.0
    light_yaw: float = 0.85
    light_pitch: float = 0.95
    latlong: np.ndarray | None = None
    finishes: np.ndarray | None = None
    flags: int = 0
    ext: abi.gr_material_ext | None = None
    _keep: list = field(default_factory=list, repr=False)

    def c_scene(self) -> abi.gr_scene:
        s = abi.gr_scene()
        s.camera = self.cam
        s.width, s.height, s.max_bounces = self.width, self.height, self.max_bounces
        planes = np.ascontiguousarray(self.planes, np.float32).reshape(-1, 4)
        self._keep = [planes]
        s.n_planes = planes.shape[0]
        s.planes = planes.ctypes.data_as(C.POINTER(abi.gr_plane)) if planes.size else None
        if self.finishes is not None:
            fin = np.ascontiguousarray(self.finishes, np.uint32)
            self._keep.append(fin)
            s.finishes = fin.ctypes.data_as(C.POINTER(C.c_uint32))
        s.material = C.pointer(self.material)
        self._keep.append(s.material)
        if self.ext is not None:
            s.material_ext = C.pointer(self.ext)
            self._keep.append(s.material_ext)
        s.env.mode = self.env_mode
        s.env.uniform_rgb[:] = [float(x) for x in self.uniform_rgb]
        temp, spot = LIGHTING_PRESETS[self.preset]
        s.env.temp_k, s.env.spot_mult = temp, spot
        s.env.exposure, s.env.light_yaw, s.env.light_pitch = self.exposure, self.light_yaw, self.light_pitch
        if self.env_mode == abi.GR_ENV_LATLONG:
            m = np.ascontiguousarray(self.latlong, np.float32)
            self._keep.append(m)
            s.env.latlong_rgb = m.ctypes.data_as(C.POINTER(C.c_float))
            s.env.latlong_h, s.env.latlong_w = m.shape[0], m.shape[1]
        s.flags = self.flags
        self._c = s
        return s
