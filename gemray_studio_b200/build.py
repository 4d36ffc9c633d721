"""Build the CUDA engine in-tree: gemray_studio_b200/libgemray_cuda.so (sm_100a).

The library is compiled with nvcc directly (no JIT cache): the .so sits next to this
file so it travels with the repository snapshot.  Floating-point flags are part of the
engine's contract with the reference arithmetic: no FMA contraction (--fmad=false on
the device, -ffp-contract=off on the host), IEEE division and square root, no fast
math.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "libgemray_cuda.so"
SOURCES = ["gr_host.cu", "gr_batch.cu", "gr_batch_classes.cu", "gr_serve.cu", "gr_stream.cu", "gr_denoise.cu",
           "gr_tonemap.cu", "gr_metrics.cu", "gr_static.cu", "gr_verify.cu", "gr_stokes.cu", "gr_single_clear.cu",
           "gr_single_general.cu", "gr_scene_builders.cpp"]
HEADERS = ["gr_device.cuh", "gr_stage.cuh", "gr_trace.cuh", "gr_launch.cuh", "gr_kernels.cuh", "gr_transport.cuh",
           "gr_single.cuh", "gr_sorted.cuh", "gr_batch.cuh",
           "gr_ctx.h", "gr_host.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Compile-time engine options (see csrc/gr_device.cuh).
DEFINES: tuple[str, ...] = ()


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def flags(extra_ptxas: bool = False) -> list[str]:
    f = [
        *ARCH, "-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
        "-ftz=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math", "-I", str(ROOT / "include"),
        "-I", str(CSRC),
    ]
    if extra_ptxas:
        f += ["-Xptxas", "-v"]
    return f


def needs_build() -> bool:
    if not OUT.exists():
        return True
    newest = max((CSRC / n).stat().st_mtime for n in SOURCES + HEADERS)
    newest = max(newest, (ROOT / "include" / "gemray_cuda.h").stat().st_mtime, Path(__file__).stat().st_mtime)
    return OUT.stat().st_mtime < newest


def build(force: bool = False, verbose: bool = False, defines: tuple[str, ...] = DEFINES, out: Path | None = None) -> Path:
    """Compile every translation unit to an object in parallel (one nvcc per source,
    objects under _build/), then link the shared library."""
    from concurrent.futures import ThreadPoolExecutor
    target = Path(out) if out is not None else OUT
    if out is None and not force and not needs_build():
        return OUT
    objdir = ROOT / "_build" / (target.stem + "".join(f"_{d}" for d in defines).replace("=", "-"))
    objdir.mkdir(parents=True, exist_ok=True)
    base = [nvcc(), *flags(verbose), *[f"-D{d}" for d in defines]]

    def compile_one(src: str):
        obj = objdir / (src.rsplit(".", 1)[0] + ".o")
        return src, subprocess.run([*base, "-c", "-o", str(obj), str(CSRC / src)], capture_output=True, text=True), obj

    jobs = max(1, min(len(SOURCES), os.cpu_count() or 1))
    with ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(compile_one, SOURCES))
    for src, r, _ in results:
        if verbose or r.returncode != 0:
            sys.stderr.write(f"--- {src}\n" + r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed compiling {src}")
    tmp = target.with_suffix(".so.tmp")
    r = subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *[str(o) for _, _, o in results]],
                       capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libgemray_cuda.so")
    os.replace(tmp, target)
    return target


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
