// torch.ops.torchscience_b200.gamma_log_likelihood_value_and_grad / _hvp:
// host side of the fused Gamma log-likelihood kernels (ops_likelihood.cu).
// Operands are promoted to a common floating dtype and broadcast; each is
// passed to the kernel as a contiguous tensor of the broadcast shape or as a
// broadcast scalar, the two layouts the kernels take.
#include <ATen/native/TypeProperties.h>
#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>
#include <torch/library.h>

#include <array>

#include "pointwise.h"

namespace tsbh {
namespace {

int32_t ll_dtype(at::ScalarType t) {
  switch (t) {
    case at::kFloat: return TSB_F32;
    case at::kDouble: return TSB_F64;
    case at::kHalf: return TSB_F16;
    case at::kBFloat16: return TSB_BF16;
    default: TORCH_CHECK(false, "torchscience_b200: unsupported dtype ", t);
  }
}

// A contiguous tensor of `shape`, or a one-element tensor seen with stride 0.
tsb_tensor ll_describe(const at::Tensor& t, at::IntArrayRef shape, at::Tensor& keep) {
  tsb_tensor d{};
  d.ndim = static_cast<int32_t>(shape.size());
  for (int i = 0; i < d.ndim; ++i) d.sizes[i] = shape[i];
  if (!t.defined()) return d;
  d.dtype = ll_dtype(t.scalar_type());
  if (t.numel() == 1) {
    keep = t.reshape({});
    d.data = keep.data_ptr();
    return d;  // strides stay 0
  }
  keep = t.expand(shape).contiguous();
  d.data = keep.data_ptr();
  int64_t s = 1;
  for (int i = d.ndim - 1; i >= 0; --i) {
    d.strides[i] = s;
    s *= shape[i];
  }
  return d;
}

void ll_check(int32_t st, const char* name) {
  TORCH_CHECK(st == TSB_OK, "torchscience_b200 ", name, ": ", tsb_status_string(st), ": ", tsb_last_error());
}

}  // namespace

std::tuple<at::Tensor, at::Tensor, at::Tensor, at::Tensor> gamma_log_likelihood_value_and_grad(
    const at::Tensor& x, const at::Tensor& shape, const at::Tensor& scale, std::array<bool, 3> grad_mask) {
  constexpr const char* name = "gamma_log_likelihood_value_and_grad";
  const at::ScalarType dt = checked_common_dtype(name, {x, shape, scale});
  const at::Device dev = checked_device(name, {x, shape, scale});
  c10::cuda::CUDAGuard guard(dev);
  auto ins = prepare_inputs({x, shape, scale}, dt, dev);
  at::DimVector full = at::infer_size_dimvector(ins[0].sizes(), ins[1].sizes());
  full = at::infer_size_dimvector(full, ins[2].sizes());
  const auto opts = ins[0].options();
  at::Tensor value = at::empty({}, opts);
  std::vector<at::Tensor> grads(3);
  for (int i = 0; i < 3; ++i)
    if (grad_mask[i]) grads[i] = at::empty(full, opts);
  std::vector<at::Tensor> keep(3), keep_out(4);
  std::vector<tsb_tensor> din(3), dout(4);
  for (int i = 0; i < 3; ++i) din[i] = ll_describe(ins[i], full, keep[i]);
  dout[0] = ll_describe(value, full, keep_out[0]);
  for (int i = 0; i < 3; ++i) dout[i + 1] = ll_describe(grads[i], full, keep_out[i + 1]);
  const int64_t wsb = tsb_gamma_log_likelihood_workspace_bytes();
  ll_check(wsb < 0 ? (int32_t)wsb : TSB_OK, name);
  at::Tensor ws = at::empty({wsb}, opts.dtype(at::kByte));
  const auto stream = c10::cuda::getCurrentCUDAStream(dev.index()).stream();
  ll_check(tsb_gamma_log_likelihood_value_and_grad(din.data(), 3, dout.data(), 4, precision_mode().load(),
                                                   ws.data_ptr(), wsb, stream),
           name);
  return {value, grads[0], grads[1], grads[2]};
}

std::tuple<at::Tensor, at::Tensor, at::Tensor> gamma_log_likelihood_hvp(
    const at::Tensor& grad, const at::Tensor& x, const at::Tensor& shape, const at::Tensor& scale,
    const std::optional<at::Tensor>& u_x, const std::optional<at::Tensor>& u_shape,
    const std::optional<at::Tensor>& u_scale, std::array<bool, 3> out_mask) {
  constexpr const char* name = "gamma_log_likelihood_hvp";
  std::vector<at::Tensor> all{grad, x, shape, scale};
  for (const auto* u : {&u_x, &u_shape, &u_scale}) all.push_back(u->has_value() ? **u : at::Tensor());
  std::vector<at::Tensor> present;
  for (const auto& t : all)
    if (t.defined()) present.push_back(t);
  const at::ScalarType dt = checked_common_dtype(name, present);
  const at::Device dev = checked_device(name, present);
  c10::cuda::CUDAGuard guard(dev);
  auto ins = prepare_inputs(present, dt, dev);
  std::vector<at::Tensor> cast(7);
  for (size_t i = 0, j = 0; i < all.size(); ++i)
    if (all[i].defined()) cast[i] = ins[j++];
  at::DimVector full(cast[1].sizes().begin(), cast[1].sizes().end());
  for (const auto& t : cast)
    if (t.defined()) full = at::infer_size_dimvector(full, t.sizes());
  const auto opts = cast[1].options();
  std::vector<at::Tensor> outs(3);
  for (int i = 0; i < 3; ++i)
    if (out_mask[i]) outs[i] = at::empty(full, opts);
  std::vector<at::Tensor> keep(7), keep_out(3);
  std::vector<tsb_tensor> din(7), dout(3);
  for (int i = 0; i < 7; ++i) din[i] = ll_describe(cast[i], full, keep[i]);
  for (int i = 0; i < 3; ++i) dout[i] = ll_describe(outs[i], full, keep_out[i]);
  int64_t numel = 1;
  for (auto v : full) numel *= v;
  if (numel == 0) return {outs[0], outs[1], outs[2]};
  const auto stream = c10::cuda::getCurrentCUDAStream(dev.index()).stream();
  ll_check(tsb_gamma_log_likelihood_hvp(din.data(), 7, dout.data(), 3, precision_mode().load(), nullptr, 0, stream),
           name);
  return {outs[0], outs[1], outs[2]};
}

}  // namespace tsbh

TORCH_LIBRARY_FRAGMENT(torchscience_b200, m) {
  m.def("gamma_log_likelihood_value_and_grad(Tensor x, Tensor shape, Tensor scale, bool[3] grad_mask) -> "
        "(Tensor, Tensor, Tensor, Tensor)");
  m.def("gamma_log_likelihood_hvp(Tensor grad, Tensor x, Tensor shape, Tensor scale, Tensor? u_x, Tensor? u_shape, "
        "Tensor? u_scale, bool[3] out_mask) -> (Tensor, Tensor, Tensor)");
}

TORCH_LIBRARY_IMPL(torchscience_b200, CUDA, m) {
  m.impl("gamma_log_likelihood_value_and_grad", tsbh::gamma_log_likelihood_value_and_grad);
  m.impl("gamma_log_likelihood_hvp", tsbh::gamma_log_likelihood_hvp);
}
