"""Framework behaviour on the GPU: broadcasting, strides, dtypes, scalars, empty
and odd sizes, >8-dim fallback, precision mode, error paths, determinism."""

import numpy as np
import pytest
import torch

import torchscience_b200 as tsb
from torchscience_b200 import special_functions as sf
from tests._util import run

pytestmark = pytest.mark.gpu
dev = "cuda"


@pytest.mark.parametrize("n", [1, 31, 33, 1023, 1025, 4097, 65537])
def test_odd_sizes_match_fp64_reference_values(n):
    x = torch.linspace(0.05, 40, n, device=dev, dtype=torch.float64)
    y = sf.log_gamma(x)
    assert torch.allclose(y, torch.lgamma(x), rtol=1e-14, atol=1e-14)
    a = torch.linspace(0.1, 30, n, device=dev, dtype=torch.float64)
    p = sf.regularized_gamma_p(a, x)
    assert torch.allclose(p, torch.special.gammainc(a, x), rtol=1e-12, atol=1e-14)


def test_broadcast_shapes_and_noncontiguous_inputs():
    a = torch.rand(5, 1, 7, device=dev, dtype=torch.float64) * 10 + 0.1
    x = torch.rand(3, 7, device=dev, dtype=torch.float64).t()[:, :1] * 10  # (7,1) -> non-contiguous
    x = x.t().expand(3, 7)  # stride-0 rows
    want = torch.special.gammainc(a, x)
    got = sf.regularized_gamma_p(a, x)
    assert got.shape == (5, 3, 7)
    assert torch.allclose(got, want, rtol=1e-12, atol=1e-14)
    z = torch.rand(64, 64, device=dev, dtype=torch.float64)[::3, ::2] * 20 + 0.1
    assert torch.allclose(sf.digamma(z), torch.special.digamma(z), rtol=1e-13, atol=1e-14)


def test_cpu_scalar_with_cuda_tensor_and_promotion():
    x = torch.rand(10, device=dev, dtype=torch.float32) * 5 + 0.1
    a = torch.tensor(2.0, dtype=torch.float64)  # 0-dim CPU tensor
    y = sf.regularized_gamma_p(a, x)
    assert y.device.type == "cuda" and y.dtype == torch.float32  # 0-dim does not promote
    y64 = sf.regularized_gamma_p(torch.full((10,), 2.0, device=dev, dtype=torch.float64), x)
    assert y64.dtype == torch.float64


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
def test_half_precision_storage(dtype):
    x = (torch.rand(1000, device=dev) * 10 + 0.5).to(dtype)
    y = sf.log_gamma(x)
    assert y.dtype == dtype
    want = torch.lgamma(x.double()).to(dtype)
    assert torch.allclose(y.double(), want.double(), rtol=1e-2, atol=1e-2)


def test_empty_and_zero_dim():
    e = torch.empty(0, 3, device=dev, dtype=torch.float64)
    assert sf.log_gamma(e).shape == (0, 3)
    s = torch.tensor(0.5, device=dev, dtype=torch.float64)
    assert abs(sf.log_gamma(s).item() - 0.5 * np.log(np.pi)) < 1e-15


def test_more_than_eight_dims_fallback():
    x = torch.rand(*([2] * 10), device=dev, dtype=torch.float64).permute(*reversed(range(10))) * 5 + 0.1
    assert torch.allclose(sf.trigamma(x), torch.special.polygamma(1, x), rtol=1e-13)


def test_precision_mode_fp64_for_float32():
    x = torch.rand(4096, device=dev) * 20 + 0.01
    with tsb.precision("fp64"):
        y64 = sf.digamma(x)
    want = torch.special.digamma(x.double()).float()
    assert torch.equal(y64, want) or (y64 - want).abs().max().item() <= 2 * torch.finfo(torch.float32).eps * want.abs().max().item()


def test_device_mismatch_raises():
    if torch.cuda.device_count() < 1:
        pytest.skip()
    with pytest.raises(RuntimeError):
        sf.regularized_gamma_p(torch.ones(3, device=dev), torch.ones(3))


def test_outputs_do_not_alias_and_are_deterministic():
    x = torch.rand(1 << 16, device=dev, dtype=torch.float64) * 30
    a = torch.rand(1 << 16, device=dev, dtype=torch.float64) * 30 + 0.01
    p1 = sf.regularized_gamma_p(a, x)
    p2 = sf.regularized_gamma_p(a, x)
    assert torch.equal(p1, p2) and p1.data_ptr() != p2.data_ptr()


def test_c_abi_reports_launch_errors_as_status_not_crash():
    """Misaligned output pointer -> TSB_ERR_ARGUMENT, nothing launched."""
    x = torch.rand(16, device=dev, dtype=torch.float64)
    buf = torch.empty(17 * 8, dtype=torch.uint8, device=dev)
    bad = buf[1:129].view(torch.uint8)  # misaligned byte offset
    from tests._util import TsbTensor, lib
    import ctypes

    din = (TsbTensor * 1)()
    din[0].data, din[0].dtype, din[0].ndim = x.data_ptr(), 1, 1
    din[0].sizes[0], din[0].strides[0] = 16, 1
    dout = (TsbTensor * 1)()
    dout[0].data, dout[0].dtype, dout[0].ndim = bad.data_ptr(), 1, 1
    dout[0].sizes[0], dout[0].strides[0] = 16, 1
    st = lib().tsb_log_gamma(din, 1, dout, 1, 0, None, ctypes.c_int64(0), None)
    assert st == -1 and b"misaligned" in lib().tsb_last_error()


@pytest.mark.parametrize("op", ["bessel_j", "modified_bessel_k", "regularized_gamma_p"])
def test_gradient_of_one_input_only(op):
    """Only the second input requires grad (the common case for Bessel
    functions of a fixed order): the first input's gradient is neither
    computed nor returned, and the second matches the full backward."""
    import numpy as np

    from torchscience_b200 import special_functions as sf

    fn = getattr(sf, op)
    first = torch.tensor([0.5, 1.5, 2.25, 3.0], dtype=torch.float64, device="cuda")
    second = torch.tensor([0.3, 1.7, 4.2, 9.0], dtype=torch.float64, device="cuda", requires_grad=True)
    y = fn(first, second)
    (g,) = torch.autograd.grad(y.sum(), second)
    full = getattr(torch.ops.torchscience, op + "_backward")(torch.ones_like(y), first, second.detach())
    np.testing.assert_array_equal(g.cpu().numpy(), full[1].cpu().numpy())
    first_rg = first.clone().requires_grad_(True)
    y2 = fn(first_rg, second.detach())
    (g2,) = torch.autograd.grad(y2.sum(), first_rg)
    assert torch.isfinite(g2).all()


def test_hyp2f1_gradient_of_z_only():
    from torchscience_b200 import special_functions as sf

    a = torch.tensor([0.7, 1.3], dtype=torch.float64, device="cuda")
    z = torch.tensor([0.2, -1.5], dtype=torch.float64, device="cuda", requires_grad=True)
    y = sf.hypergeometric_2_f_1(a, a + 0.5, a + 2.0, z)
    (gz,) = torch.autograd.grad(y.sum(), z, create_graph=True)
    (gzz,) = torch.autograd.grad(gz.sum(), z)
    assert torch.isfinite(gz).all() and torch.isfinite(gzz).all()
