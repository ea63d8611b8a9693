"""Reports elements whose series, continued fraction or recurrence stopped at
its iteration cap.

Every loop in the kernels is bounded, so an input that would need more terms
than the cap costs time but never hangs; its result is then a truncated sum.
The kernels count such elements per device (a counter the loops touch only
when they reach the cap); reading the count waits for the device.
"""

from __future__ import annotations

import contextlib
import warnings

import torch


class ConvergenceWarning(RuntimeWarning):
    """Some elements stopped at their iteration cap."""


def unconverged_count(device=None, reset: bool = False) -> int:
    """Elements that reached an iteration cap on `device` (default: the
    current CUDA device) since the last reset; waits for the device."""
    index = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    return int(torch.ops.torchscience_b200.unconverged_count(index.index or 0, reset))


@contextlib.contextmanager
def check_convergence(action: str = "warn", device=None):
    """Resets the count on entry and, on exit, warns (action="warn") or raises
    RuntimeError (action="raise") if any element of the enclosed calls
    reached an iteration cap."""
    if action not in ("warn", "raise"):
        raise ValueError(f"action must be 'warn' or 'raise', got {action!r}")
    unconverged_count(device, reset=True)
    yield
    n = unconverged_count(device, reset=True)
    if n:
        msg = f"{n} element(s) stopped at an iteration cap; their results are truncated sums"
        if action == "raise":
            raise RuntimeError(msg)
        warnings.warn(msg, ConvergenceWarning, stacklevel=3)
