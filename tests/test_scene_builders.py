"""The product's scene builders (libgemray_cuda.so: Camera::new, the standard round
brilliant, the 13 built-in materials) agree bit for bit with the oracle's independent
restatement of the same reference code."""
from __future__ import annotations

import ctypes as C

import numpy as np

from gemray_studio_b200 import abi, scene as S


def test_standard_round_brilliant_matches_oracle(oracle, engine_lib):
    buf = (abi.gr_plane * 128)()
    n = oracle.gro_standard_round_brilliant(buf, 128)
    ref = np.ctypeslib.as_array(buf).view(np.float32).reshape(-1, 4)[:n]
    got = S.standard_round_brilliant()
    assert got.shape == (74, 4)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    # every normal is unit length and the solid contains the origin
    assert np.allclose(np.linalg.norm(got[:, :3], axis=1), 1.0, atol=1e-6)
    assert np.all(got[:, 3] < 0)


def test_builtin_materials_match_oracle(oracle, engine_lib):
    for name in S.BUILTIN_MATERIALS:
        a = abi.gr_material()
        assert oracle.gro_builtin_material(name.encode(), C.byref(a)) == 0
        b = S.builtin_material(name)
        assert bytes(a) == bytes(b), name
    assert engine_lib.gr_builtin_material(b"Unobtainium", C.byref(abi.gr_material())) == abi.GR_ENOTFOUND


def test_camera_matches_oracle(oracle, engine_lib):
    for args in [(0.35, 0.28, 5.0, 18.0), (0.0, 0.45, 4.0, 42.0), (1.1, 1.5707, 3.0, 30.0), (2.0, 0.0, 6.0, 25.0)]:
        a = abi.gr_camera()
        oracle.gro_camera_new(*args, C.byref(a))
        b = S.camera(*args)
        assert bytes(a) == bytes(b), args


def test_synthetic_geometry_is_valid():
    for planes in (S.round_brilliant_57(), S.emerald_cut_49(), S.random_polyhedron(np.random.default_rng(3))):
        assert planes.ndim == 2 and planes.shape[1] == 4
        assert np.allclose(np.linalg.norm(planes[:, :3], axis=1), 1.0, atol=1e-6)
        assert np.all(planes[:, 3] < 0), "origin must be strictly inside every half-space"
    assert S.emerald_cut_49().shape[0] == 49
    assert S.face_count(S.emerald_cut_49()) == 49          # every plane bounds a face
    assert S.face_count(S.round_brilliant_57()) == 73      # 57 facets + 16 girdle planes
    assert S.face_count(S.standard_round_brilliant()) == 74


def test_custom_material_matches_new_custom_encoding():
    """GemMaterial::new_custom (optics/materials.rs:1257-1316) as GpuGemMaterial::encode
    writes it: Cauchy a = n_d - b / 0.5893^2 with b = dispersion x k_FC, c-axis +Y,
    trigonal + uniaxial-positive above |dn| > 1e-4, legacy RGB bands on both modes."""
    import numpy as np

    from gemray_studio_b200 import abi, scene as S
    m = S.custom_material(1.5, 0.0, 0.03)
    d = m.dispersion
    assert d.model_type == abi.GR_DISP_CAUCHY and d.param_a[0] == np.float32(1.5) and d.param_a[1] == 0.0
    assert list(d.c_axis_and_birefringence) == [0.0, 1.0, 0.0, np.float32(0.03)]
    assert d.is_anisotropic == 1 and m.crystal_system == 3 and m.optical_character == 1
    assert m.o_ray_band_count == 3 and m.o_ray_bands[0].center_nm == 620.0 and m.e_ray_bands[2].width_nm == 45.0
    assert m.beta_ray_band_count == 0 and m.beta_ray_bands[0].width_nm == 1.0 and m.absorption_path_scale == 1.0
    iso = S.custom_material(2.417, 0.044, 0.0)
    f = np.float32
    k = f(1) / (f(1) / (f(0.4861) * f(0.4861)) - f(1) / (f(0.6563) * f(0.6563)))
    b = f(0.044) * k
    assert iso.dispersion.param_a[1] == b and iso.dispersion.param_a[0] == f(2.417) - b / (f(0.5893) * f(0.5893))
    assert iso.dispersion.is_anisotropic == 0 and iso.crystal_system == 0 and iso.optical_character == 0
