"""Builds the two native libraries of torchscience_b200 in-tree.

libtsb_cuda.so  the sm_100a kernels behind the C ABI in include/torchscience_b200.h
                (nvcc only; no torch dependency).
libtsb_ops.so   the torch.ops.torchscience registration (CUDA / Meta / Autograd /
                AutocastCUDA / CPU-error kernels) that calls the C ABI.

Usage: python torchscience_b200/_build.py [--force] [-j N]
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
KERNELS = PKG / "csrc" / "kernels"
HOST = PKG / "csrc" / "host"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH_FLAGS + [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "--expt-relaxed-constexpr",
    f"-I{INCLUDE}",
]

KERNEL_LIB = PKG / "libtsb_cuda.so"
OPS_LIB = PKG / "libtsb_ops.so"


def _newest(paths) -> float:
    return max((p.stat().st_mtime for p in paths), default=0.0)


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout)
        raise RuntimeError(f"command failed ({proc.returncode}): {' '.join(cmd[:6])} ...")


def _deps_of(obj: Path):
    """Headers the unit included when `obj` was last compiled (the compiler's
    -MD dependency file beside it), or None when there is no such record."""
    dfile = obj.with_suffix(".d")
    if not dfile.exists():
        return None
    text = dfile.read_text().replace("\\\n", " ")
    _, _, rest = text.partition(":")
    return [Path(t) for t in rest.split()]


def _compile_units(units, out_dir: Path, compile_fn, deps_mtime: float, force: bool, jobs: int):
    """Compiles each unit whose object is missing or older than the unit or
    any header it included (from its dependency file; without one, older
    than any header of the tree, `deps_mtime`)."""
    out_dir.mkdir(parents=True, exist_ok=True)
    todo, objs = [], []
    for src in units:
        obj = out_dir / (src.stem + ".o")
        objs.append(obj)
        deps = _deps_of(obj) if obj.exists() else None
        if deps is None or not all(d.exists() for d in deps):
            newest = deps_mtime
        else:
            newest = _newest(deps)
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest):
            todo.append((src, obj))
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            futs = [ex.submit(compile_fn, s, o) for s, o in todo]
            for f in futs:
                f.result()
    return objs, bool(todo)


def build_kernels(force: bool = False, jobs: int | None = None) -> Path:
    jobs = jobs or os.cpu_count() or 4
    units = sorted(KERNELS.glob("*.cu"))
    deps = _newest(list(KERNELS.glob("*.cuh")) + list(INCLUDE.glob("*.h")))

    def cc(src, obj):
        _run([NVCC, *NVCC_FLAGS, "-MD", "-MF", str(obj.with_suffix(".d")), "-c", str(src), "-o", str(obj)])

    objs, changed = _compile_units(units, BUILD / "kernels", cc, deps, force, jobs)
    for stale in (BUILD / "kernels").glob("*.o"):
        if stale not in objs:  # a unit that was removed or renamed
            stale.unlink()
            stale.with_suffix(".d").unlink(missing_ok=True)
    if changed or force or not KERNEL_LIB.exists() or KERNEL_LIB.stat().st_mtime < _newest(objs):
        _run([NVCC, *ARCH_FLAGS, "-shared", "-o", str(KERNEL_LIB), *map(str, objs), "-Xcompiler", "-fPIC"])
    return KERNEL_LIB


def _torch_flags():
    import torch
    from torch.utils import cpp_extension

    inc = cpp_extension.include_paths()
    libdir = cpp_extension.library_paths()[0]
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cflags = [f"-I{p}" for p in inc] + [
        f"-I{CUDA_HOME / 'include'}",
        f"-I{INCLUDE}",
        f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
        "-DUSE_C10D_NCCL",
    ]
    ldflags = [
        f"-L{libdir}",
        "-lc10",
        "-lc10_cuda",
        "-ltorch",
        "-ltorch_cpu",
        "-ltorch_cuda",
        f"-Wl,-rpath,{libdir}",
    ]
    return cflags, ldflags


def build_ops(force: bool = False, jobs: int | None = None) -> Path:
    jobs = jobs or os.cpu_count() or 4
    cflags, ldflags = _torch_flags()
    units = sorted(HOST.glob("*.cpp"))
    deps = _newest(list(HOST.glob("*.h")) + list(INCLUDE.glob("*.h")))

    def cc(src, obj):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", *cflags, "-MD", "-MF", str(obj.with_suffix(".d")), "-c", str(src),
              "-o", str(obj)])

    objs, changed = _compile_units(units, BUILD / "host", cc, deps, force, jobs)
    if changed or force or not OPS_LIB.exists() or OPS_LIB.stat().st_mtime < max(_newest(objs), KERNEL_LIB.stat().st_mtime):
        _run(
            [
                "g++",
                "-shared",
                "-o",
                str(OPS_LIB),
                *map(str, objs),
                f"-L{PKG}",
                "-ltsb_cuda",
                "-Wl,-rpath,$ORIGIN",
                *ldflags,
            ]
        )
    return OPS_LIB


def build(force: bool = False, jobs: int | None = None) -> None:
    build_kernels(force, jobs)
    build_ops(force, jobs)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    build(a.force, a.j)
    print(f"built {KERNEL_LIB.name} and {OPS_LIB.name}")
