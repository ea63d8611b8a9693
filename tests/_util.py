"""Shared test helpers: error metrics, fixtures and the C-ABI binding."""

from __future__ import annotations

import os

import numpy as np
import torch

from torchscience_b200._cabi import TsbTensor, call, describe, header_entry_points, lib, run  # noqa: F401

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")

def rel_err(got, want, floor=1e-300):
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        e = np.abs(got - want) / np.maximum(np.abs(want), floor)
    both_nan = np.isnan(got) & np.isnan(want)
    same_inf = np.isinf(got) & np.isinf(want) & (np.sign(got) == np.sign(want))
    e = np.where(both_nan | same_inf, 0.0, e)
    return e


def ulp_err(got, want):
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    u = np.spacing(np.abs(want))
    with np.errstate(invalid="ignore"):
        e = np.abs(got - want) / u
    both_nan = np.isnan(got) & np.isnan(want)
    same_inf = np.isinf(got) & np.isinf(want) & (np.sign(got) == np.sign(want))
    return np.where(both_nan | same_inf, 0.0, e)


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name + ".npz"))
