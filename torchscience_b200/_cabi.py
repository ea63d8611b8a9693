"""ctypes binding of the C ABI (include/torchscience_b200.h) over torch tensors.

Lets Python code call the sm_100a kernels directly, without the
torch.ops.torchscience registration: used by the tests and by bench.py to time
individual kernels on the launching stream.
"""

from __future__ import annotations

import ctypes
import os
import re

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
KERNEL_LIB = os.path.join(_HERE, "libtsb_cuda.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "torchscience_b200.h")

TSB_MAX_DIMS = 8
DTYPES = {torch.float32: 0, torch.float64: 1, torch.float16: 2, torch.bfloat16: 3}


class TsbTensor(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("dtype", ctypes.c_int32),
        ("ndim", ctypes.c_int32),
        ("sizes", ctypes.c_int64 * TSB_MAX_DIMS),
        ("strides", ctypes.c_int64 * TSB_MAX_DIMS),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(KERNEL_LIB)
        _lib.tsb_last_error.restype = ctypes.c_char_p
        _lib.tsb_status_string.restype = ctypes.c_char_p
        _lib.tsb_version.restype = ctypes.c_char_p
        _lib.tsb_workspace_bytes.restype = ctypes.c_int64
        _lib.tsb_launch_count.restype = ctypes.c_int64
    return _lib


def header_entry_points() -> list[str]:
    text = open(HEADER).read()
    ops = re.findall(r"^TSB_OP_SIGNATURE\((tsb_\w+)\);", text, re.M)
    funcs = re.findall(r"^(?:const char\*|int64_t|int32_t)\s+(tsb_\w+)\(", text, re.M)
    return ops + funcs


def describe(t: torch.Tensor | None, shape) -> TsbTensor:
    d = TsbTensor()
    d.ndim = len(shape)
    for i, s in enumerate(shape):
        d.sizes[i] = s
    if t is None:
        d.data = None
        d.dtype = 0
        return d
    v = t.expand(shape)
    d.data = t.data_ptr()
    d.dtype = DTYPES[t.dtype]
    for i in range(len(shape)):
        d.strides[i] = v.stride(i)
    return d


def call(name: str, inputs, outputs, precision: int = 0, workspace: torch.Tensor | None = None, shape=None) -> int:
    """Calls tsb_<name> through the C ABI on the current stream; returns the status."""
    if shape is None:
        shape = torch.broadcast_shapes(*[t.shape for t in inputs])
    shape = tuple(shape)
    din = (TsbTensor * len(inputs))(*[describe(t, shape) for t in inputs])
    dout = (TsbTensor * len(outputs))(*[describe(t, shape) for t in outputs])
    fn = getattr(lib(), "tsb_" + name)
    ws = ctypes.c_void_p(workspace.data_ptr()) if workspace is not None else ctypes.c_void_p(None)
    wsb = workspace.numel() if workspace is not None else 0
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream) if torch.cuda.is_available() else None
    return fn(din, len(inputs), dout, len(outputs), precision, ws, ctypes.c_int64(wsb), stream)


def sweep_scratch_bytes(shape) -> int:
    """Bytes of the workspace that only the row-sorted sweep of a 2-D grid
    uses (its row order, row and column tables of 16 doubles per entry, one
    32-bit column mask per 32 x 32 task, and the task counters): the last part
    of what tsb_workspace_bytes asks for on such a grid."""
    n0, n1 = (shape[-2], shape[-1]) if len(shape) >= 2 else (0, 0)
    tasks = ((n0 + 31) // 32) * ((n1 + 31) // 32)
    return (((max(n0, n1) * 4 + 255) & ~255) + (((n0 + n1) * 16 * 8 + 255) & ~255) + ((tasks * 4 + 255) & ~255)
            + 256)


def run(name: str, *inputs, n_out: int = 1, precision: int = 0, out_shapes=None, sweep: bool = True) -> list[torch.Tensor]:
    """Broadcast call through the C ABI; outputs full-shape unless out_shapes
    given (reduced).  The workspace is the one tsb_workspace_bytes asks for;
    with sweep=False it is cut short of the sweep's scratch (none at all when
    no output is reduced), so a 2-D grid runs the unsorted tile kernel."""
    shape = torch.broadcast_shapes(*[t.shape for t in inputs])
    outs = []
    for k in range(n_out):
        s = shape if out_shapes is None or out_shapes[k] is None else out_shapes[k]
        outs.append(torch.empty(s, dtype=inputs[0].dtype, device=inputs[0].device))
    din = (TsbTensor * len(inputs))(*[describe(t, shape) for t in inputs])
    dout = (TsbTensor * n_out)(*[describe(o, shape) for o in outs])
    nbytes = lib().tsb_workspace_bytes(din, len(inputs), dout, n_out)
    assert nbytes >= 0, lib().tsb_last_error()
    reduced = out_shapes is not None and any(s is not None and tuple(s) != tuple(shape) for s in out_shapes)
    if not sweep and nbytes > 0:
        nbytes = nbytes - sweep_scratch_bytes(shape) if reduced else 0
    ws = torch.empty(nbytes, dtype=torch.uint8, device=inputs[0].device) if nbytes > 0 else None
    st = call(name, list(inputs), outs, precision=precision, workspace=ws, shape=shape)
    assert st == 0, f"tsb_{name} -> {st}: {lib().tsb_last_error().decode()}"
    return outs
