"""C ABI checks that need no GPU: exports, status strings, argument validation."""

import ctypes

import numpy as np
import pytest
import torch

from tests._util import TsbTensor, header_entry_points, lib

FAKE = 0x100000  # aligned, never dereferenced by validation paths


def desc(shape, strides=None, dtype=1, data=FAKE):
    d = TsbTensor()
    d.ndim = len(shape)
    d.dtype = dtype
    d.data = data
    if strides is None:
        strides = [int(np.prod(shape[i + 1 :])) for i in range(len(shape))]
    for i, (s, st) in enumerate(zip(shape, strides)):
        d.sizes[i] = s
        d.strides[i] = st
    return d


def arr(*ds):
    return (TsbTensor * len(ds))(*ds)


def test_every_declared_symbol_is_exported():
    names = header_entry_points()
    assert len(names) >= 28
    L = lib()
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/torchscience_b200.h but not exported"


def test_version_and_status_strings():
    L = lib()
    assert b"sm_100a" in L.tsb_version()
    for st, word in [(0, b"ok"), (-1, b"argument"), (-2, b"dtype"), (-3, b"layout"), (-4, b"workspace"), (-5, b"launch"), (-6, b"device")]:
        assert word in L.tsb_status_string(st)


def test_wrong_operand_count_is_rejected_before_any_launch():
    L = lib()
    st = L.tsb_log_gamma(arr(desc([8]), desc([8])), 2, arr(desc([8])), 1, 0, None, ctypes.c_int64(0), None)
    assert st == -1 and b"expected 1 inputs" in L.tsb_last_error()


def test_null_input_and_mixed_dtype_are_rejected():
    L = lib()
    st = L.tsb_regularized_gamma_p(arr(desc([8], data=None), desc([8])), 2, arr(desc([8])), 1, 0, None, ctypes.c_int64(0), None)
    assert st == -1
    st = L.tsb_regularized_gamma_p(arr(desc([8], dtype=0), desc([8], dtype=1)), 2, arr(desc([8])), 1, 0, None, ctypes.c_int64(0), None)
    assert st == -2


def test_bad_precision_and_shape_mismatch():
    L = lib()
    st = L.tsb_log_gamma(arr(desc([8])), 1, arr(desc([8])), 1, 7, None, ctypes.c_int64(0), None)
    assert st == -1
    st = L.tsb_log_gamma(arr(desc([8])), 1, arr(desc([9])), 1, 0, None, ctypes.c_int64(0), None)
    assert st == -1


def test_empty_iteration_is_a_no_op():
    L = lib()
    st = L.tsb_log_gamma(arr(desc([0])), 1, arr(desc([0])), 1, 0, None, ctypes.c_int64(0), None)
    assert st == 0


def test_workspace_query_for_the_broadcast_grid():
    L = lib()
    shape = [4096, 4096]
    g = desc(shape)
    a = desc(shape, strides=[1, 0])
    x = desc(shape, strides=[0, 1])
    ga = desc(shape, strides=[1, 0])
    gx = desc(shape, strides=[0, 1])
    n = L.tsb_workspace_bytes(arr(g, a, x), 3, arr(ga, gx), 2)
    # row-reduced: 128 column tiles x 4096 rows; column-reduced: 128 row tiles (32 rows) x 4096 cols (doubles);
    # then the row-sorted sweep's scratch: the row order (4096 int32), row and column tables (16 doubles per
    # row and per column), one 32-bit column mask per task of 32 x 32 elements, and the task counters (256 bytes)
    sweep = 4096 * 4 + (4096 + 4096) * 16 * 8 + 128 * 128 * 4 + 256
    assert n == (128 + 128) * 4096 * 8 + sweep
    # no reduced output: only the sweep's scratch on an (R, 1) x (1, C) grid
    assert L.tsb_workspace_bytes(arr(g, a, x), 3, arr(desc(shape), desc(shape)), 2) == sweep
    # ... and nothing for a layout without a row-constant and a column-constant input
    assert L.tsb_workspace_bytes(arr(g, g, g), 3, arr(desc(shape), desc(shape)), 2) == 0


def test_reduced_layout_needing_three_dims_is_reported():
    L = lib()
    shape = [4, 5, 6]
    g = desc(shape)
    a = desc(shape, strides=[6, 0, 1])  # (4,1,6)
    x = desc(shape, strides=[0, 1, 0])  # (1,5,1)
    ga = desc(shape, strides=[6, 0, 1])
    assert L.tsb_workspace_bytes(arr(g, a, x), 3, arr(ga, desc(shape, data=None)), 2) == -3


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device path")
def test_valid_call_without_a_device_reports_device_error():
    L = lib()
    st = L.tsb_log_gamma(arr(desc([8])), 1, arr(desc([8])), 1, 0, None, ctypes.c_int64(0), None)
    assert st == -6


def test_launch_counter_is_exported_and_starts_without_launches():
    n = lib().tsb_launch_count()
    assert n >= 0
    # An empty iteration launches nothing.
    from tests._util import TsbTensor

    t = TsbTensor()
    t.data, t.dtype, t.ndim = None, 1, 1
    t.sizes[0] = 0
    o = TsbTensor()
    o.data, o.dtype, o.ndim = None, 1, 1
    o.sizes[0] = 0
    lib().tsb_log_gamma((TsbTensor * 1)(t), 1, (TsbTensor * 1)(o), 1, 0, None, 0, None)
    assert lib().tsb_launch_count() == n
