"""torchscience_b200: sm_100a (B200) kernels for torchscience's special functions.

Importing the package loads the native libraries, which register the
``torch.ops.torchscience.*`` operators (same names and schemas as the
reference's ``torchscience._csrc``) for CUDA, Meta, Autograd and AutocastCUDA.
The Python-level API lives in :mod:`torchscience_b200.special_functions` with
the reference's function names.  There is no CPU fallback: CPU tensors raise.
"""

from __future__ import annotations

import os as _os

import torch as _torch

_HERE = _os.path.dirname(_os.path.abspath(__file__))
KERNEL_LIBRARY = _os.path.join(_HERE, "libtsb_cuda.so")
OPS_LIBRARY = _os.path.join(_HERE, "libtsb_ops.so")

if not (_os.path.exists(KERNEL_LIBRARY) and _os.path.exists(OPS_LIBRARY)):
    raise ImportError(
        "torchscience_b200 native libraries are not built "
        f"(expected {OPS_LIBRARY}); run `python torchscience_b200/_build.py`"
    )

_torch.ops.load_library(OPS_LIBRARY)

from . import probability, special_functions  # noqa: E402
from ._convergence import ConvergenceWarning, check_convergence, unconverged_count  # noqa: E402
from ._precision import (  # noqa: E402
    autograd_strategy,
    get_autograd_strategy,
    get_precision_mode,
    precision,
    set_autograd_strategy,
    set_precision_mode,
)

__all__ = [
    "probability",
    "special_functions",
    "set_precision_mode",
    "get_precision_mode",
    "precision",
    "set_autograd_strategy",
    "get_autograd_strategy",
    "autograd_strategy",
    "unconverged_count",
    "check_convergence",
    "ConvergenceWarning",
    "KERNEL_LIBRARY",
    "OPS_LIBRARY",
]
