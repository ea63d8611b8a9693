"""Precision mode for float32 / float16 / bfloat16 data, and the autograd
strategy of regularized_gamma_p / regularized_gamma_q.

"mixed" (default): FP32 arithmetic for the bulk of each evaluation, FP64 only
in the classified regions that need it.  "fp64": the FP64 kernels for every
dtype (results rounded to the input dtype).  float64 data always uses the FP64
kernels.  The mode is process-wide; ``TORCHSCIENCE_B200_PRECISION`` sets the
initial value.
"""

from __future__ import annotations

import contextlib
import os

import torch

_MODES = {"mixed": 0, "auto": 0, "fp64": 1}
_NAMES = {0: "mixed", 1: "fp64"}


def set_precision_mode(mode: str) -> str:
    """Sets the mode ("mixed" or "fp64"); returns the previous one."""
    if mode not in _MODES:
        raise ValueError(f"precision mode must be one of {sorted(_MODES)}, got {mode!r}")
    prev = torch.ops.torchscience_b200.set_precision_mode(_MODES[mode])
    return _NAMES[int(prev)]


def get_precision_mode() -> str:
    return _NAMES[int(torch.ops.torchscience_b200.get_precision_mode())]


@contextlib.contextmanager
def precision(mode: str):
    """Context manager form of :func:`set_precision_mode`."""
    prev = set_precision_mode(mode)
    try:
        yield
    finally:
        set_precision_mode(prev)


_env = os.environ.get("TORCHSCIENCE_B200_PRECISION")
if _env:
    set_precision_mode(_env.strip().lower())


_STRATEGIES = ("keep", "recompute")


def set_autograd_strategy(strategy: str) -> str:
    """How autograd differentiates regularized_gamma_p / _q on CUDA; returns
    the previous strategy.

    "keep" (default): the recorded forward evaluates the value and both first
    derivatives in one pass and keeps the derivatives (16 bytes per element of
    float64 output stay alive until the backward, which only multiplies them
    by the incoming gradient).  "recompute": the forward evaluates the value
    alone and the backward evaluates the derivatives again from the inputs,
    reducing them to the inputs' shapes in the same pass (no extra memory).
    ``TORCHSCIENCE_B200_AUTOGRAD`` sets the initial value.
    """
    if strategy not in _STRATEGIES:
        raise ValueError(f"autograd strategy must be one of {_STRATEGIES}, got {strategy!r}")
    prev = torch.ops.torchscience_b200.set_keep_derivatives(strategy == "keep")
    return "keep" if prev else "recompute"


def get_autograd_strategy() -> str:
    return "keep" if torch.ops.torchscience_b200.get_keep_derivatives() else "recompute"


@contextlib.contextmanager
def autograd_strategy(strategy: str):
    """Context manager form of :func:`set_autograd_strategy`."""
    prev = set_autograd_strategy(strategy)
    try:
        yield
    finally:
        set_autograd_strategy(prev)


_env = os.environ.get("TORCHSCIENCE_B200_AUTOGRAD")
if _env:
    set_autograd_strategy(_env.strip().lower())
