// Host glue between ATen tensors and the torchscience_b200 C ABI.
#pragma once

#include <ATen/ATen.h>
#include <ATen/TensorIterator.h>

#include <atomic>
#include <string>
#include <vector>

#include "torchscience_b200.h"

namespace tsbh {

using OpFn = int32_t (*)(const tsb_tensor*, int32_t, const tsb_tensor*, int32_t, int32_t, void*, int64_t, void*);

// Process-wide precision mode for f32/f16/bf16 data (TSB_PRECISION_AUTO:
// mixed kernels; TSB_PRECISION_FP64: FP64 kernels).  f64 data always uses
// the FP64 kernels.
std::atomic<int>& precision_mode();

// Common dtype of `inputs` with TensorIterator's promotion rules; raises
// NotImplementedError for integral/bool and complex dtypes, mirroring the
// reference's AT_DISPATCH_FLOATING_TYPES_AND2(BFloat16, Half) dispatch
// (cpu/macros.h:963).
at::ScalarType checked_common_dtype(const char* name, at::TensorList inputs);

// Device of the first CUDA input; CPU 0-dim tensors are moved to it; any
// other CPU tensor is an error (there is no CPU fallback).
at::Device checked_device(const char* name, at::TensorList inputs);

// Inputs cast to `dtype` and moved to `device`.
std::vector<at::Tensor> prepare_inputs(at::TensorList inputs, at::ScalarType dtype, at::Device device);

// Broadcast pointwise call: outputs get the broadcast shape (allocated by
// TensorIterator, like the reference's CPU path), every output computed.
std::vector<at::Tensor> run_pointwise(OpFn fn, const char* name, at::TensorList inputs, int n_out);

// Backward with gradients reduced to the inputs' own shapes.  `grad_inputs`
// are the forward inputs whose gradients are wanted (want[i]); the result
// has one tensor per forward input (undefined where not wanted).  Uses the
// fused reduction of the C ABI when the layout allows, otherwise full-shape
// gradients summed with at::sum_to.
std::vector<at::Tensor> run_reduced_backward(OpFn fn, const char* name, const at::Tensor& grad,
                                             at::TensorList fwd_inputs, const std::vector<bool>& want);

// run_pointwise computing only the outputs with want[o] set (the others come
// back undefined; the kernel skips them).
std::vector<at::Tensor> run_pointwise_masked(OpFn fn, const char* name, at::TensorList inputs, int n_out,
                                             const std::vector<bool>& want);

// General form of run_reduced_backward: `kernel_inputs` go to the kernel as
// they are (broadcast together), output i is reduced to out_like[i]'s shape.
std::vector<at::Tensor> run_reduced(OpFn fn, const char* name, at::TensorList kernel_inputs, at::TensorList out_like,
                                    const std::vector<bool>& want);

// Meta (shape/dtype only) version of run_pointwise.
std::vector<at::Tensor> meta_pointwise(const char* name, at::TensorList inputs, int n_out);

// Raises the reference-style error for CPU tensors.
[[noreturn]] void cpu_not_supported(const char* name);

}  // namespace tsbh
