"""The allocation-free regularized_gamma_p backward, through the C ABI.

tsb_regularized_gamma_p_backward_noalloc serves callers that cannot allocate
device memory (hosts that reach the library only through a C FFI and own no
device allocator, loops that must not call cudaMalloc because it can
synchronize the device): it keeps the partial sums of the reduced gradients
in a fixed file-scope device array instead of a caller workspace.  Its
results must equal those of tsb_regularized_gamma_p_backward with a
workspace, call after call (the array keeps the previous call's contents).
This file is collected last so that a failure here cannot hide other tests;
it also passes on its own in a fresh process (the first call does the
per-device set-up).
"""

import ctypes

import numpy as np
import pytest
import torch

import torchscience_b200  # noqa: F401  (loads the libraries)
from torchscience_b200._cabi import TsbTensor, describe, lib, run

pytestmark = pytest.mark.gpu

NOALLOC_SCRATCH_BYTES = 8 << 20  # TSB_NOALLOC_SCRATCH_BYTES


def noalloc(g, a, x, ga, gx):
    shape = tuple(torch.broadcast_shapes(g.shape, a.shape, x.shape))
    din = (TsbTensor * 3)(describe(g, shape), describe(a, shape), describe(x, shape))
    dout = (TsbTensor * 2)(describe(ga, shape), describe(gx, shape))
    fn = lib().tsb_regularized_gamma_p_backward_noalloc
    fn.restype = ctypes.c_int32
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return fn(din, 3, dout, 2, 0, stream)


def inputs(seed, rows, cols, dtype):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    a = torch.exp(torch.empty(rows, 1, device="cuda", dtype=torch.float64).uniform_(np.log(1e-2), np.log(1e3), generator=gen))
    x = torch.exp(torch.empty(1, cols, device="cuda", dtype=torch.float64).uniform_(np.log(1e-3), np.log(2e3), generator=gen))
    g = torch.randn(rows, cols, device="cuda", dtype=torch.float64, generator=gen)
    return a.to(dtype), x.to(dtype), g.to(dtype)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-5)])
def test_noalloc_matches_the_workspace_entry_point_on_two_calls(dtype, tol):
    for call, (seed, rows, cols) in enumerate([(0, 1000, 777), (1, 513, 2049)]):
        a, x, g = inputs(seed, rows, cols, dtype)
        want_a, want_x = run("regularized_gamma_p_backward", g, a, x, n_out=2, out_shapes=[a.shape, x.shape])
        ga = torch.full_like(a, float("nan"))
        gx = torch.full_like(x, float("nan"))
        st = noalloc(g, a, x, ga, gx)
        assert st == 0, f"call {call}: {lib().tsb_last_error().decode()}"
        torch.cuda.synchronize()
        for got, want in ((ga, want_a), (gx, want_x)):
            scale = want.double().abs().max().item()
            assert torch.allclose(got.double(), want.double(), rtol=tol, atol=tol * scale), f"call {call}"


@pytest.mark.parametrize("layout", ["scalar_a", "full_shape"])
def test_noalloc_other_layouts(layout):
    """A scalar a reduces its gradient over the whole grid (one partial per
    tile in the scratch array); full-shape a and x need no scratch at all."""
    a, x, g = inputs(2, 300, 517, torch.float64)
    if layout == "scalar_a":
        a = a[:1, :1].clone()  # (1, 1): broadcast along both dimensions
    else:
        a, x = a.expand(g.shape).contiguous(), x.expand(g.shape).contiguous()
    for call in range(2):
        want_a, want_x = run("regularized_gamma_p_backward", g, a, x, n_out=2, out_shapes=[a.shape, x.shape])
        ga = torch.full_like(a, float("nan"))
        gx = torch.full_like(x, float("nan"))
        st = noalloc(g, a, x, ga, gx)
        assert st == 0, f"call {call}: {lib().tsb_last_error().decode()}"
        torch.cuda.synchronize()
        for got, want in ((ga, want_a), (gx, want_x)):
            scale = want.double().abs().max().item()
            assert torch.allclose(got.double(), want.double(), rtol=1e-12, atol=1e-12 * scale), f"call {call}"


def test_noalloc_rejects_requests_beyond_its_scratch():
    # 70000 rows x 4096 columns: the row-reduced partials alone need
    # 128 column tiles x 70000 rows x 8 bytes, far above 8 MiB.  The upstream
    # gradient is broadcast from one element, so the test allocates little.
    a = torch.full((70000, 1), 2.0, device="cuda", dtype=torch.float64)
    x = torch.full((1, 4096), 1.5, device="cuda", dtype=torch.float64)
    g = torch.ones(1, 1, device="cuda", dtype=torch.float64).expand(70000, 4096)
    ga, gx = torch.empty_like(a), torch.empty_like(x)
    st = noalloc(g, a, x, ga, gx)
    assert st == -4  # TSB_ERR_WORKSPACE
    assert b"scratch" in lib().tsb_last_error()
