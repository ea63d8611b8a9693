#include "pointwise.h"

#include <ATen/native/TypeProperties.h>
#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>

namespace tsbh {

std::atomic<int>& precision_mode() {
  static std::atomic<int> mode{TSB_PRECISION_AUTO};
  return mode;
}

namespace {

int32_t to_tsb_dtype(at::ScalarType t) {
  switch (t) {
    case at::kFloat: return TSB_F32;
    case at::kDouble: return TSB_F64;
    case at::kHalf: return TSB_F16;
    case at::kBFloat16: return TSB_BF16;
    case at::kComplexFloat: return TSB_C64;
    case at::kComplexDouble: return TSB_C128;
    default: TORCH_CHECK(false, "torchscience_b200: unsupported dtype ", t);
  }
}

// Operators with complex64 / complex128 kernels (and their backward and
// double-backward ops).
bool takes_complex(const char* name) {
  static const char* const ops[] = {"log_gamma", "gamma", "digamma", "trigamma", "log_beta", "beta"};
  const std::string n(name);
  for (const char* op : ops) {
    const std::string o(op);
    if (n == o || n == o + "_backward" || n == o + "_backward_backward") return true;
  }
  return false;
}

// Descriptor of `t` viewed over the iteration shape `shape` (t must be
// broadcastable to it; broadcast dims get stride 0).
tsb_tensor describe(const at::Tensor& t, at::IntArrayRef shape, bool present = true) {
  tsb_tensor d{};
  d.ndim = static_cast<int32_t>(shape.size());
  d.dtype = present ? to_tsb_dtype(t.scalar_type()) : TSB_F32;
  d.data = present ? t.data_ptr() : nullptr;
  if (!present) {
    for (int i = 0; i < d.ndim; ++i) d.sizes[i] = shape[i];
    return d;
  }
  const at::Tensor v = t.expand(shape);
  for (int i = 0; i < d.ndim; ++i) {
    d.sizes[i] = shape[i];
    d.strides[i] = v.stride(i);
  }
  return d;
}

void check_status(int32_t st, const char* name) {
  TORCH_CHECK(st == TSB_OK, "torchscience_b200 ", name, ": ", tsb_status_string(st), ": ", tsb_last_error());
}

// Calls `fn` with the workspace the C ABI asks for (none for most layouts;
// for a (R, 1) x (1, C) grid, the row order of the sorted sweep), taken from
// the caching allocator on the current stream.
void call_with_workspace(OpFn fn, const char* name, std::vector<tsb_tensor>& din, std::vector<tsb_tensor>& dout,
                         const at::TensorOptions& opts, cudaStream_t stream) {
  const int64_t ws = tsb_workspace_bytes(din.data(), (int32_t)din.size(), dout.data(), (int32_t)dout.size());
  check_status(ws < 0 ? (int32_t)ws : TSB_OK, name);
  at::Tensor workspace;
  if (ws > 0) workspace = at::empty({ws}, opts.dtype(at::kByte));
  check_status(fn(din.data(), (int32_t)din.size(), dout.data(), (int32_t)dout.size(), precision_mode().load(),
                  ws > 0 ? workspace.data_ptr() : nullptr, ws, stream),
               name);
}

}  // namespace

[[noreturn]] void cpu_not_supported(const char* name) {
  TORCH_CHECK(false, "torchscience_b200: \"", name,
              "\" runs on CUDA tensors only; got CPU tensors (this build has no CPU fallback)");
}

at::ScalarType checked_common_dtype(const char* name, at::TensorList inputs) {
  at::native::ResultTypeState state = {};
  for (const auto& t : inputs) state = at::native::update_result_type_state(t, state);
  const at::ScalarType dt = at::native::result_type(state);
  if (at::isComplexType(dt)) {
    TORCH_CHECK_NOT_IMPLEMENTED(takes_complex(name), "\"", name, "\" not implemented for '", c10::toString(dt),
                                "' in torchscience_b200 (complex dtypes: log_gamma, gamma, digamma, trigamma, log_beta, beta)");
    TORCH_CHECK_NOT_IMPLEMENTED(dt == at::kComplexFloat || dt == at::kComplexDouble, "\"", name,
                                "\" not implemented for '", c10::toString(dt), "'");
    return dt;
  }
  TORCH_CHECK_NOT_IMPLEMENTED(at::isFloatingType(dt), "\"", name, "\" not implemented for '", c10::toString(dt), "'");
  TORCH_CHECK_NOT_IMPLEMENTED(dt == at::kFloat || dt == at::kDouble || dt == at::kHalf || dt == at::kBFloat16, "\"",
                              name, "\" not implemented for '", c10::toString(dt), "'");
  return dt;
}

at::Device checked_device(const char* name, at::TensorList inputs) {
  for (const auto& t : inputs)
    if (t.defined() && t.is_cuda()) return t.device();
  cpu_not_supported(name);
}

std::vector<at::Tensor> prepare_inputs(at::TensorList inputs, at::ScalarType dtype, at::Device device) {
  std::vector<at::Tensor> out;
  out.reserve(inputs.size());
  for (const auto& t : inputs) {
    at::Tensor u = t;
    if (u.device() != device) {
      TORCH_CHECK(u.dim() == 0 && u.is_cpu(), "torchscience_b200: expected all tensors on ", device, ", got ",
                  u.device());
      u = u.to(device);
    }
    if (u.scalar_type() != dtype) u = u.to(dtype);
    out.push_back(u);
  }
  return out;
}

std::vector<at::Tensor> run_pointwise(OpFn fn, const char* name, at::TensorList inputs, int n_out) {
  const at::ScalarType dt = checked_common_dtype(name, inputs);
  const at::Device dev = checked_device(name, inputs);
  c10::cuda::CUDAGuard guard(dev);
  std::vector<at::Tensor> ins = prepare_inputs(inputs, dt, dev);

  at::TensorIteratorConfig cfg;
  cfg.set_check_mem_overlap(true);
  std::vector<at::Tensor> outs(n_out);
  for (int o = 0; o < n_out; ++o) cfg.add_output(outs[o]);
  for (const auto& t : ins) cfg.add_const_input(t);
  at::TensorIterator iter = cfg.build();
  std::vector<at::Tensor> res;
  for (int o = 0; o < n_out; ++o) res.push_back(iter.output(o));
  if (iter.numel() == 0) return res;

  const int n_in = static_cast<int>(ins.size());
  std::vector<tsb_tensor> din(n_in), dout(n_out);
  const int nd = iter.ndim();
  const int64_t esz = c10::elementSize(dt);
  if (nd <= TSB_MAX_DIMS) {
    // TensorIterator orders dims fastest-first; the C ABI is row-major.
    auto fill = [&](tsb_tensor& d, int arg) {
      d.data = iter.data_ptr(arg);
      d.dtype = to_tsb_dtype(dt);
      d.ndim = nd;
      for (int i = 0; i < nd; ++i) {
        d.sizes[i] = iter.shape()[nd - 1 - i];
        d.strides[i] = iter.strides(arg)[nd - 1 - i] / esz;
      }
    };
    for (int o = 0; o < n_out; ++o) fill(dout[o], o);
    for (int i = 0; i < n_in; ++i) fill(din[i], n_out + i);
  } else {
    // More than TSB_MAX_DIMS non-coalescible dims: gather to dense buffers.
    const at::DimVector shape(iter.shape().rbegin(), iter.shape().rend());
    const std::vector<int64_t> flat{iter.numel()};
    std::vector<at::Tensor> dense_in;
    for (const auto& t : ins) dense_in.push_back(t.expand(res[0].sizes()).contiguous().view(flat));
    std::vector<at::Tensor> dense_out;
    for (int o = 0; o < n_out; ++o) dense_out.push_back(at::empty(flat, res[0].options()));
    for (int i = 0; i < n_in; ++i) din[i] = describe(dense_in[i], flat);
    for (int o = 0; o < n_out; ++o) dout[o] = describe(dense_out[o], flat);
    const auto stream = c10::cuda::getCurrentCUDAStream(dev.index()).stream();
    check_status(fn(din.data(), n_in, dout.data(), n_out, precision_mode().load(), nullptr, 0, stream), name);
    for (int o = 0; o < n_out; ++o) res[o].copy_(dense_out[o].view(res[o].sizes()));
    return res;
  }
  const auto stream = c10::cuda::getCurrentCUDAStream(dev.index()).stream();
  call_with_workspace(fn, name, din, dout, res[0].options(), stream);
  return res;
}

std::vector<at::Tensor> run_reduced_backward(OpFn fn, const char* name, const at::Tensor& grad,
                                             at::TensorList fwd_inputs, const std::vector<bool>& want) {
  std::vector<at::Tensor> all;
  all.push_back(grad);
  for (const auto& t : fwd_inputs) all.push_back(t);
  return run_reduced(fn, name, all, fwd_inputs, want);
}

std::vector<at::Tensor> run_reduced(OpFn fn, const char* name, at::TensorList all, at::TensorList fwd_inputs,
                                    const std::vector<bool>& want) {
  const at::ScalarType dt = checked_common_dtype(name, all);
  const at::Device dev = checked_device(name, all);
  c10::cuda::CUDAGuard guard(dev);
  std::vector<at::Tensor> ins = prepare_inputs(all, dt, dev);

  at::DimVector full(ins[0].sizes().begin(), ins[0].sizes().end());
  for (size_t i = 1; i < ins.size(); ++i) full = at::infer_size_dimvector(full, ins[i].sizes());

  const int n_fwd = static_cast<int>(fwd_inputs.size());
  std::vector<at::Tensor> grads(n_fwd);
  const auto opts = ins[0].options();
  for (int i = 0; i < n_fwd; ++i)
    if (want[i]) grads[i] = at::empty(fwd_inputs[i].sizes(), opts);

  int64_t numel = 1;
  for (auto s : full) numel *= s;
  if (numel == 0) {
    for (int i = 0; i < n_fwd; ++i)
      if (want[i]) grads[i].zero_();
    return grads;
  }
  if (full.size() > TSB_MAX_DIMS) {
    // Fall back to full-shape gradients reduced by ATen.
    auto full_grads = run_pointwise(fn, name, ins, n_fwd);
    for (int i = 0; i < n_fwd; ++i)
      if (want[i]) grads[i] = at::sum_to(full_grads[i], fwd_inputs[i].sizes());
    return grads;
  }

  std::vector<tsb_tensor> din, dout;
  for (const auto& t : ins) din.push_back(describe(t, full));
  for (int i = 0; i < n_fwd; ++i) dout.push_back(want[i] ? describe(grads[i], full) : describe(at::Tensor(), full, false));
  // Complex entry points do not reduce outputs: their broadcast gradients
  // take the full-shape path below.
  const int64_t ws = at::isComplexType(dt) ? (int64_t)TSB_ERR_LAYOUT
                                           : tsb_workspace_bytes(din.data(), (int32_t)din.size(), dout.data(),
                                                                 (int32_t)dout.size());
  if (ws == TSB_ERR_LAYOUT) {
    // Not a 2-D broadcast pattern (or complex data): full-shape gradients + sum_to.
    std::vector<at::Tensor> full_grads(n_fwd);
    std::vector<tsb_tensor> dfull;
    for (int i = 0; i < n_fwd; ++i) {
      if (want[i]) {
        full_grads[i] = at::empty(full, opts);
        dfull.push_back(describe(full_grads[i], full));
      } else {
        dfull.push_back(describe(at::Tensor(), full, false));
      }
    }
    const auto stream = c10::cuda::getCurrentCUDAStream(dev.index()).stream();
    check_status(fn(din.data(), (int32_t)din.size(), dfull.data(), n_fwd, precision_mode().load(), nullptr, 0, stream),
                 name);
    for (int i = 0; i < n_fwd; ++i)
      if (want[i]) grads[i] = at::sum_to(full_grads[i], fwd_inputs[i].sizes());
    return grads;
  }
  check_status(ws < 0 ? (int32_t)ws : TSB_OK, name);
  at::Tensor workspace;
  if (ws > 0) workspace = at::empty({ws}, opts.dtype(at::kByte));
  const auto stream = c10::cuda::getCurrentCUDAStream(dev.index()).stream();
  check_status(fn(din.data(), (int32_t)din.size(), dout.data(), n_fwd, precision_mode().load(),
                  ws > 0 ? workspace.data_ptr() : nullptr, ws, stream),
               name);
  return grads;
}

std::vector<at::Tensor> run_pointwise_masked(OpFn fn, const char* name, at::TensorList inputs, int n_out,
                                             const std::vector<bool>& want) {
  const at::ScalarType dt = checked_common_dtype(name, inputs);
  const at::Device dev = checked_device(name, inputs);
  c10::cuda::CUDAGuard guard(dev);
  std::vector<at::Tensor> ins = prepare_inputs(inputs, dt, dev);
  at::DimVector full(ins[0].sizes().begin(), ins[0].sizes().end());
  for (size_t i = 1; i < ins.size(); ++i) full = at::infer_size_dimvector(full, ins[i].sizes());
  const auto opts = ins[0].options();
  std::vector<at::Tensor> res(n_out);
  for (int o = 0; o < n_out; ++o)
    if (want[o]) res[o] = at::empty(full, opts);
  int64_t numel = 1;
  for (auto v : full) numel *= v;
  if (numel == 0) return res;
  if (full.size() > TSB_MAX_DIMS) {  // every output through run_pointwise, unwanted ones dropped
    auto all = run_pointwise(fn, name, ins, n_out);
    for (int o = 0; o < n_out; ++o)
      if (want[o]) res[o] = all[o];
    return res;
  }
  std::vector<tsb_tensor> din, dout;
  for (const auto& t : ins) din.push_back(describe(t, full));
  for (int o = 0; o < n_out; ++o) dout.push_back(want[o] ? describe(res[o], full) : describe(at::Tensor(), full, false));
  const auto stream = c10::cuda::getCurrentCUDAStream(dev.index()).stream();
  call_with_workspace(fn, name, din, dout, opts, stream);
  return res;
}

std::vector<at::Tensor> meta_pointwise(const char* name, at::TensorList inputs, int n_out) {
  const at::ScalarType dt = checked_common_dtype(name, inputs);
  std::vector<at::Tensor> ins;
  for (const auto& t : inputs) ins.push_back(t.scalar_type() == dt ? t : t.to(dt));
  at::TensorIteratorConfig cfg;
  std::vector<at::Tensor> outs(n_out);
  for (int o = 0; o < n_out; ++o) cfg.add_output(outs[o]);
  for (const auto& t : ins) cfg.add_const_input(t);
  at::TensorIterator iter = cfg.build();
  std::vector<at::Tensor> res;
  for (int o = 0; o < n_out; ++o) res.push_back(iter.output(o));
  return res;
}

}  // namespace tsbh
