"""Build recipe for the oracle's native parts (test infrastructure only).

  oracle/liboracle.so             the C restatement (oracle/refalg.c); needs only gcc.
  oracle/_ref/libref_scalar.so    the reference's own scalar kernels behind a C ABI
                                  (oracle/ref_scalar_shim.cpp), compiled from the
                                  reference's headers where they lie.
  oracle/_ref/libtorchscience_ref.so
                                  the reference's own CPU torch operators for the
                                  accelerated ops (oracle/ref_ops.cpp), for the
                                  reference arm of bench.py.

The two _ref libraries are built from the reference checkout named by the
REFERENCE_ROOT environment variable; with it unset (or pointing at no
sources) they are not rebuilt, a message says so, and any existing build is
kept.  They are git-ignored build products.  Nothing is written outside
oracle/.

Usage: REFERENCE_ROOT=<reference checkout> python oracle/build_ref.py [--force]
"""

from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
REF_ROOT = Path(os.environ["REFERENCE_ROOT"]) if os.environ.get("REFERENCE_ROOT") else None
REF_CSRC = REF_ROOT / "src" / "torchscience" / "csrc" if REF_ROOT else None
OUT = HERE / "_ref"


def _run(cmd):
    p = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stdout[-8000:])
        raise RuntimeError(f"oracle build failed: {' '.join(map(str, cmd[:4]))} ...")


def _stale(target: Path, *sources: Path) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def _torch():
    import torch
    from torch.utils import cpp_extension

    return (
        Path(torch.__file__).parent,
        cpp_extension.include_paths(),
        cpp_extension.library_paths()[0],
        int(torch._C._GLIBCXX_USE_CXX11_ABI),
    )


def build_restatement(force=False) -> Path:
    src, lib = HERE / "refalg.c", HERE / "liboracle.so"
    if force or _stale(lib, src):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp", str(src), "-o", str(lib), "-lm"])
    return lib


def build_reference(force=False) -> list[Path]:
    if REF_CSRC is None or not REF_CSRC.is_dir():
        have = [p for p in (OUT / "libref_scalar.so", OUT / "libtorchscience_ref.so") if p.exists()]
        why = "REFERENCE_ROOT is unset" if REF_CSRC is None else f"no reference sources under {REF_ROOT}"
        sys.stderr.write(f"oracle/build_ref.py: {why}; oracle/_ref not rebuilt"
                         f" ({len(have)} existing librar{'y' if len(have) == 1 else 'ies'} kept)\n")
        return have
    OUT.mkdir(exist_ok=True)
    _, incs, libdir, abi = _torch()
    common = ["-std=c++17", "-fPIC", "-shared", "-fopenmp", f"-I{REF_CSRC}", f"-D_GLIBCXX_USE_CXX11_ABI={abi}"]
    import sysconfig

    common += [f"-I{p}" for p in incs] + [f"-I{sysconfig.get_paths()['include']}"]
    built = []
    shim, shim_lib = HERE / "ref_scalar_shim.cpp", OUT / "libref_scalar.so"
    if force or _stale(shim_lib, shim):
        _run(["g++", "-O3", *common, str(shim), "-o", str(shim_lib), f"-L{libdir}", "-lc10", f"-Wl,-rpath,{libdir}"])
    built.append(shim_lib)
    ops, ops_lib = HERE / "ref_ops.cpp", OUT / "libtorchscience_ref.so"
    schemas = REPO / "torchscience_b200" / "csrc" / "host" / "schemas.h"
    if force or _stale(ops_lib, ops, schemas):
        _run(
            [
                "g++",
                "-O3",
                *common,
                f"-I{schemas.parent}",
                str(ops),
                "-o",
                str(ops_lib),
                f"-L{libdir}",
                "-lc10",
                "-ltorch",
                "-ltorch_cpu",
                f"-Wl,-rpath,{libdir}",
            ]
        )
    built.append(ops_lib)
    return built


def build(force=False):
    out = [build_restatement(force)]
    out += build_reference(force)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    for p in build(a.force):
        print("built", p.relative_to(REPO))
