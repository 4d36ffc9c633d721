"""C-ABI checks that need no GPU: the library builds for sm_100a, loads, exports every
entry point include/gemray_cuda.h declares, the struct layouts agree, and the
failure contract holds (no device => GR_NO_DEVICE, never an abort)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from gemray_studio_b200 import abi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "gemray_cuda.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*[A-Za-z_][\w \*]*?\b(gr_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_compiles_with_static_asserts():
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-x", "c++", str(HEADER)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run(["gcc", "-std=c11", "-fsyntax-only", "-x", "c", str(HEADER)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def header_int_constants() -> dict[str, int]:
    """Every `#define GR_* <integer expression>` of the header, evaluated."""
    out = {}
    for name, expr in re.findall(r"^#define\s+(GR_\w+)\s+(.+?)\s*(?:/\*.*)?$", HEADER.read_text(), flags=re.M):
        py = re.sub(r"(?<=[0-9a-fA-F])[uU][lL]*\b", "", expr)
        if not re.fullmatch(r"[0-9a-fA-Fx()<>| +\-*]+", py):
            continue
        out[name] = eval(py, {"__builtins__": {}})
    return out


def test_python_constants_match_header():
    consts = header_int_constants()
    assert "GR_KERNEL_AUTO" in consts and consts["GR_AUTO_STAGED_MIN_TUPLES"] == 1 << 19
    shared = [n for n in consts if hasattr(abi, n)]
    assert len(shared) >= 10
    for n in shared:
        assert getattr(abi, n) == consts[n], n


def test_library_exports_every_declared_symbol(engine_lib):
    names = declared_functions()
    assert len(names) >= 15
    nm = subprocess.run(["nm", "-D", "--defined-only", str(abi.library_path())], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (gr_\w+)", nm))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        getattr(engine_lib, n)  # resolvable through ctypes
    # the ctypes mirror declares every header entry point
    assert {e[0] for e in abi.EXPORTS} == set(names)


def test_library_is_built_for_sm100a(engine_lib):
    """The build compiles device code for sm_100a only (the runtime check of the loaded
    cubin is tests/test_gpu_case_banks.py::test_device_code_is_sm100)."""
    from gemray_studio_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "-gencode" in build.flags() and "arch=compute_100a,code=sm_100a" in build.flags()


def test_struct_layouts_match_header():
    src = r'''
#include <cstdio>
#include <cstddef>
#include "gemray_cuda.h"
int main(){ printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(gr_scene), offsetof(gr_scene, planes),
 offsetof(gr_scene, env), sizeof(gr_environment), offsetof(gr_environment, latlong_rgb), sizeof(gr_material_ext),
 sizeof(gr_rng_record), sizeof(gr_create_opts)); }
'''
    tmp = Path("/tmp/gr_layout.cpp")
    tmp.write_text(src)
    exe = Path("/tmp/gr_layout")
    subprocess.run(["g++", "-I", str(ROOT / "include"), str(tmp), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    want = [C.sizeof(abi.gr_scene), abi.gr_scene.planes.offset, abi.gr_scene.env.offset, C.sizeof(abi.gr_environment),
            abi.gr_environment.latlong_rgb.offset, C.sizeof(abi.gr_material_ext), C.sizeof(abi.gr_rng_record),
            C.sizeof(abi.gr_create_opts)]
    assert got == want


def test_create_without_device_reports_no_device(engine_lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    ctx = C.c_void_p()
    st = engine_lib.gr_create(C.byref(ctx), None)
    assert st == abi.GR_NO_DEVICE
    assert not ctx.value
    assert engine_lib.gr_last_error_string()
    assert engine_lib.gr_destroy(None) == abi.GR_OK


def test_null_arguments_are_rejected(engine_lib):
    assert engine_lib.gr_create(None, None) == abi.GR_EINVAL
    assert engine_lib.gr_accumulate(None, None, 0, 1, None) == abi.GR_EINVAL
    assert engine_lib.gr_set_kernel(None, 0) == abi.GR_EINVAL


def test_backend_acquire_without_device_declines(engine_lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    import numpy as np
    from gemray_studio_b200 import GpuBackend
    from helpers import srb_scene
    b = GpuBackend.acquire()
    assert b.adapter_label() is None
    sc = srb_scene(width=4, height=4)
    acc = np.zeros((16, 3), np.float32)
    assert b.try_accumulate(sc, 0, 4, acc) is False
    assert not acc.any()
    with pytest.raises(ValueError):
        b.try_accumulate(sc, 0, 4, np.zeros((15, 3), np.float32))
    assert GpuBackend.disabled().try_accumulate(sc, 0, 4, acc) is False
