"""Host-layer checks that need no GPU: schemas, Meta kernels, errors, autograd plumbing."""

import pytest
import torch

import torchscience_b200 as tsb
from torchscience_b200 import special_functions as sf

# The reference's schema strings (src/torchscience/csrc/torchscience.cpp:813-1021).
REFERENCE_SCHEMAS = [
    "gamma(Tensor z) -> Tensor",
    "gamma_backward(Tensor grad_output, Tensor z) -> Tensor",
    "gamma_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "digamma(Tensor z) -> Tensor",
    "trigamma(Tensor z) -> Tensor",
    "log_gamma(Tensor z) -> Tensor",
    "log_gamma_backward(Tensor grad_output, Tensor z) -> Tensor",
    "log_gamma_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "regularized_gamma_p(Tensor a, Tensor x) -> Tensor",
    "regularized_gamma_p_backward(Tensor grad, Tensor a, Tensor x) -> (Tensor, Tensor)",
    "regularized_gamma_p_backward_backward(Tensor grad_grad_a, Tensor grad_grad_x, Tensor grad, Tensor a, Tensor x) -> (Tensor, Tensor, Tensor)",
    "regularized_gamma_q(Tensor a, Tensor x) -> Tensor",
    "bessel_j_0(Tensor z) -> Tensor",
    "spherical_bessel_j(Tensor n, Tensor z) -> Tensor",
    "spherical_bessel_j_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor, Tensor)",
    "spherical_bessel_y(Tensor n, Tensor z) -> Tensor",
    "spherical_bessel_y_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor, Tensor)",
    "spherical_bessel_i(Tensor n, Tensor z) -> Tensor",
    "spherical_bessel_i_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor, Tensor)",
    "spherical_bessel_k(Tensor n, Tensor z) -> Tensor",
    "spherical_bessel_k_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor, Tensor)",
    "spherical_bessel_j_0(Tensor z) -> Tensor",
    "spherical_bessel_j_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "spherical_bessel_j_1(Tensor z) -> Tensor",
    "spherical_bessel_j_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "spherical_bessel_y_0(Tensor z) -> Tensor",
    "spherical_bessel_y_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "spherical_bessel_y_1(Tensor z) -> Tensor",
    "spherical_bessel_y_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "spherical_bessel_i_0(Tensor z) -> Tensor",
    "spherical_bessel_i_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "spherical_bessel_i_1(Tensor z) -> Tensor",
    "spherical_bessel_i_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "spherical_bessel_k_0(Tensor z) -> Tensor",
    "spherical_bessel_k_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "spherical_bessel_k_1(Tensor z) -> Tensor",
    "spherical_bessel_k_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "bessel_j_1(Tensor z) -> Tensor",
    "bessel_j_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "bessel_y_0(Tensor z) -> Tensor",
    "bessel_y_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "bessel_y_1(Tensor z) -> Tensor",
    "bessel_y_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "modified_bessel_i_0(Tensor z) -> Tensor",
    "modified_bessel_i_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "modified_bessel_i_1(Tensor z) -> Tensor",
    "modified_bessel_i_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "modified_bessel_k_0(Tensor z) -> Tensor",
    "modified_bessel_k_0_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "modified_bessel_k_1(Tensor z) -> Tensor",
    "modified_bessel_k_1_backward_backward(Tensor gg_z, Tensor grad_output, Tensor z) -> (Tensor, Tensor)",
    "beta(Tensor a, Tensor b) -> Tensor",
    "beta_backward_backward(Tensor gg_a, Tensor gg_b, Tensor grad_output, Tensor a, Tensor b) -> (Tensor, Tensor, Tensor)",
    "polygamma(Tensor n, Tensor z) -> Tensor",
    "polygamma_backward_backward(Tensor gg_n, Tensor gg_z, Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor, Tensor)",
    "log_beta(Tensor a, Tensor b) -> Tensor",
    "log_beta_backward(Tensor grad_output, Tensor a, Tensor b) -> (Tensor, Tensor)",
    "bessel_j(Tensor n, Tensor z) -> Tensor",
    "bessel_j_backward(Tensor grad_output, Tensor n, Tensor z) -> (Tensor, Tensor)",
    "bessel_y(Tensor n, Tensor z) -> Tensor",
    "modified_bessel_i(Tensor n, Tensor z) -> Tensor",
    "modified_bessel_k(Tensor n, Tensor z) -> Tensor",
    "incomplete_beta(Tensor x, Tensor a, Tensor b) -> Tensor",
    "incomplete_beta_backward(Tensor grad_output, Tensor x, Tensor a, Tensor b) -> (Tensor, Tensor, Tensor)",
    "incomplete_beta_backward_backward(Tensor gg_x, Tensor gg_a, Tensor gg_b, Tensor grad_output, Tensor x, Tensor a, Tensor b) -> (Tensor, Tensor, Tensor, Tensor)",
    "hypergeometric_2_f_1(Tensor a, Tensor b, Tensor c, Tensor z) -> Tensor",
    "hypergeometric_2_f_1_backward(Tensor grad_output, Tensor a, Tensor b, Tensor c, Tensor z) -> (Tensor, Tensor, Tensor, Tensor)",
    "complete_legendre_elliptic_integral_k(Tensor m) -> Tensor",
    "complete_legendre_elliptic_integral_e_backward_backward(Tensor gg_m, Tensor grad_output, Tensor m) -> (Tensor, Tensor)",
    # probability callers (torchscience.cpp:1881-1924)
    "chi2_cumulative_distribution(Tensor x, Tensor df) -> Tensor",
    "chi2_cumulative_distribution_backward(Tensor grad, Tensor x, Tensor df) -> (Tensor, Tensor)",
    "gamma_cumulative_distribution(Tensor x, Tensor shape, Tensor scale) -> Tensor",
    "gamma_cumulative_distribution_backward(Tensor grad, Tensor x, Tensor shape, Tensor scale) -> (Tensor, Tensor, Tensor)",
    "poisson_cumulative_distribution(Tensor k, Tensor rate) -> Tensor",
    "poisson_cumulative_distribution_backward(Tensor grad, Tensor k, Tensor rate) -> (Tensor, Tensor)",
    "chi2_survival(Tensor x, Tensor df) -> Tensor",
    "chi2_survival_backward(Tensor grad, Tensor x, Tensor df) -> (Tensor, Tensor)",
    "chi2_probability_density(Tensor x, Tensor df) -> Tensor",
    "chi2_probability_density_backward(Tensor grad, Tensor x, Tensor df) -> (Tensor, Tensor)",
    "gamma_probability_density(Tensor x, Tensor shape, Tensor scale) -> Tensor",
    "gamma_probability_density_backward(Tensor grad, Tensor x, Tensor shape, Tensor scale) -> (Tensor, Tensor, Tensor)",
]


@pytest.mark.parametrize("schema", REFERENCE_SCHEMAS)
def test_schema_strings_match_the_reference(schema):
    name = schema.split("(")[0]
    op = getattr(torch.ops.torchscience, name).default
    assert str(op._schema) == "torchscience::" + schema


def meta(*shape, dtype=torch.float32, rg=False):
    return torch.empty(*shape, device="meta", dtype=dtype, requires_grad=rg)


def test_meta_broadcast_and_promotion():
    y = sf.regularized_gamma_p(meta(4, 1), meta(1, 5, dtype=torch.float64))
    assert y.shape == (4, 5) and y.dtype == torch.float64
    y = sf.log_gamma(meta(3, 2, dtype=torch.bfloat16))
    assert y.shape == (3, 2) and y.dtype == torch.bfloat16
    ga, gx = torch.ops.torchscience.regularized_gamma_p_backward(meta(4, 5), meta(4, 1), meta(1, 5))
    assert ga.shape == (4, 5) and gx.shape == (4, 5)
    a, b = torch.ops.torchscience.log_gamma_backward_backward(meta(7), meta(7), meta(7))
    assert a.shape == b.shape == (7,)


def test_integer_and_complex_inputs_raise_not_implemented():
    with pytest.raises(NotImplementedError, match="Long"):
        sf.log_gamma(torch.empty(3, dtype=torch.long, device="meta"))
    # complex dtypes: the gamma and beta families have kernels; the other operators raise
    with pytest.raises(NotImplementedError, match="complex dtypes"):
        sf.bessel_j_0(torch.empty(3, dtype=torch.complex64, device="meta"))
    for fn in (sf.log_gamma, sf.gamma, sf.digamma, sf.trigamma):
        for dt in (torch.complex64, torch.complex128):
            y = fn(torch.empty(3, dtype=dt, device="meta"))
            assert y.shape == (3,) and y.dtype == dt


def test_cpu_tensors_raise_no_fallback():
    with pytest.raises(RuntimeError, match="CUDA tensors only"):
        sf.regularized_gamma_p(torch.ones(3), torch.ones(3))
    with pytest.raises(RuntimeError, match="CUDA tensors only"):
        torch.ops.torchscience.digamma_backward(torch.ones(3), torch.ones(3))


def test_autograd_plumbing_on_meta_reduces_broadcast_grads():
    a = meta(4, 1, dtype=torch.float64, rg=True)
    x = meta(1, 5, dtype=torch.float64, rg=True)
    y = sf.regularized_gamma_p(a, x)
    ga, gx = torch.autograd.grad(y.sum(), (a, x), create_graph=True)
    assert ga.shape == a.shape and gx.shape == x.shape
    (gaa,) = torch.autograd.grad(ga.sum(), (a,))
    assert gaa.shape == a.shape


def test_autograd_requires_grad_flags_respected():
    a = meta(3, dtype=torch.float64)
    x = meta(3, dtype=torch.float64, rg=True)
    y = sf.regularized_gamma_q(a, x)
    (gx,) = torch.autograd.grad(y.sum(), (x,))
    assert gx.shape == x.shape


def test_precision_mode_api():
    assert tsb.get_precision_mode() == "mixed"
    with tsb.precision("fp64"):
        assert tsb.get_precision_mode() == "fp64"
    assert tsb.get_precision_mode() == "mixed"
    with pytest.raises(ValueError):
        tsb.set_precision_mode("fp16")


def test_probability_meta_shapes_and_reduced_gradients():
    from torchscience_b200 import probability as pb

    x = meta(5, 1, rg=True)
    sh = meta(1, 3, rg=True)
    sc = meta(1, rg=True)
    y = pb.gamma_cumulative_distribution(x, sh, sc)
    assert y.shape == (5, 3) and y.device.type == "meta"
    gx, gs, gc = torch.autograd.grad(y.sum(), (x, sh, sc))
    assert gx.shape == x.shape and gs.shape == sh.shape and gc.shape == sc.shape
    assert pb.chi2_cumulative_distribution(meta(4, dtype=torch.float64), 3.0).dtype == torch.float64
    assert pb.poisson_cumulative_distribution(meta(2, 1), meta(6)).shape == (2, 6)
