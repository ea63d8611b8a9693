"""ORACLE — test infrastructure only.

ctypes loaders for the CPU checkers:

* :func:`restated` — the plain-C restatement of the reference's algorithms
  (oracle/refalg.c -> oracle/liboracle.so).
* :func:`reference` — the reference's own scalar kernels compiled from its
  sources (oracle/ref_scalar_shim.cpp -> oracle/_ref/libref_scalar.so); None
  when that library was not built (no reference sources on this machine).

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this
module; the product never imports it.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
RESTATED_LIB = HERE / "liboracle.so"
REFERENCE_LIB = HERE / "_ref" / "libref_scalar.so"
REFERENCE_OPS_LIB = HERE / "_ref" / "libtorchscience_ref.so"

_restated = None
_reference = None


def _load_restated():
    global _restated
    if _restated is None:
        if not RESTATED_LIB.exists():
            raise FileNotFoundError(f"{RESTATED_LIB} not built; run python oracle/build_ref.py")
        lib = ctypes.CDLL(str(RESTATED_LIB))
        lib.oracle_eval.argtypes = [
            ctypes.c_char_p,
            ctypes.c_int,
            ctypes.POINTER(ctypes.c_void_p),
            ctypes.POINTER(ctypes.c_void_p),
            ctypes.c_int64,
        ]
        lib.oracle_eval.restype = ctypes.c_int
        _restated = lib
    return _restated


def reference_available() -> bool:
    return REFERENCE_LIB.exists()


def _load_reference():
    global _reference
    if _reference is None:
        if not REFERENCE_LIB.exists():
            return None
        lib = ctypes.CDLL(str(REFERENCE_LIB))
        lib.ref_eval.argtypes = [
            ctypes.c_char_p,
            ctypes.c_int,
            ctypes.c_int,
            ctypes.POINTER(ctypes.c_void_p),
            ctypes.POINTER(ctypes.c_void_p),
            ctypes.c_int64,
        ]
        lib.ref_eval.restype = ctypes.c_int
        _reference = lib
    return _reference


def _pack(arrays):
    return (ctypes.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])


N_OUT = {0: 1, 1: None, 2: None}


def _n_outputs(n_inputs_fwd: int, pass_: int) -> int:
    if pass_ == 0:
        return 1
    if pass_ == 1:
        return n_inputs_fwd
    return n_inputs_fwd + 1


def restated(name: str, pass_: int, *inputs, n_out: int | None = None) -> list[np.ndarray]:
    """Evaluates the C restatement elementwise over broadcast float64 inputs."""
    lib = _load_restated()
    arrs = np.broadcast_arrays(*[np.asarray(a, dtype=np.float64) for a in inputs])
    shape = arrs[0].shape
    ins = [np.ascontiguousarray(a).ravel() for a in arrs]
    if n_out is None:
        n_out = 1 if pass_ == 0 else len(ins) - 1
    outs = [np.empty(ins[0].size) for _ in range(n_out)]
    st = lib.oracle_eval(name.encode(), pass_, _pack(ins), _pack(outs), ins[0].size)
    if st != 0:
        raise ValueError(f"oracle has no {name} pass {pass_}")
    return [o.reshape(shape) for o in outs]


def reference(name: str, pass_: int, *inputs, dtype=np.float64) -> list[np.ndarray] | None:
    """Evaluates the reference's compiled scalar kernel elementwise (None if not built)."""
    lib = _load_reference()
    if lib is None:
        return None
    arrs = np.broadcast_arrays(*[np.asarray(a, dtype=dtype) for a in inputs])
    shape = arrs[0].shape
    ins = [np.ascontiguousarray(a).ravel() for a in arrs]
    n_fwd = len(ins) if pass_ == 0 else (len(ins) - 1 if pass_ == 1 else None)
    if pass_ == 2:
        # backward_backward inputs: n gg's, grad, n forward inputs -> n + 1 outputs
        n_fwd = (len(ins) - 1) // 2
    n_out = _n_outputs(n_fwd, pass_)
    outs = [np.empty(ins[0].size, dtype=dtype) for _ in range(n_out)]
    st = lib.ref_eval(name.encode(), pass_, 1 if dtype == np.float64 else 0, _pack(ins), _pack(outs), ins[0].size)
    if st != 0:
        raise ValueError(f"reference shim has no {name} pass {pass_}")
    return [o.reshape(shape) for o in outs]


def threads() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
