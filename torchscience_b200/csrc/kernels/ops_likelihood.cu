// Fused Gamma log-likelihood: value, gradient and Hessian-vector product.
//
// For x ~ Gamma(shape k, scale θ) the log-density of one element is
//   ℓ = (k - 1) ln x - x/θ - lnΓ(k) - k ln θ
// (the logarithm of the density whose backward the reference writes in
// kernel/probability/gamma_probability_density_backward.h:11-31), with
//   ∂ℓ/∂x = (k - 1)/x - 1/θ,   ∂ℓ/∂k = ln x - ψ(k) - ln θ,   ∂ℓ/∂θ = (x/θ - k)/θ
// and the symmetric Hessian
//   ∂²/∂x² = -(k-1)/x²   ∂²/∂x∂k = 1/x    ∂²/∂x∂θ = 1/θ²
//   ∂²/∂k² = -ψ'(k)      ∂²/∂k∂θ = -1/θ   ∂²/∂θ² = (k - 2x/θ)/θ²
// (ψ' as in log_gamma_backward_backward.h:11-20).
//
// tsb_gamma_log_likelihood_value_and_grad reads x, k, θ once and writes
// L = Σ ℓ (a deterministic sum in double: per-thread, then per block in a
// fixed tree, then the block partials in block order) together with the
// requested per-element gradients, one pass: 12 bytes read and 4 to 12
// written per float element.  tsb_gamma_log_likelihood_hvp gives
// g·H·u per element for a scalar (or broadcast) g and any of u_x, u_k, u_θ.
// Float data computes in FP32 (lgammaf, and ψ, ψ' from gamma_math.cuh);
// the per-element terms are summed in double.
#include "dispatch.cuh"
#include "gamma_math.cuh"

namespace tsb {
namespace {

constexpr int kLLBlock = 256;
constexpr int kLLBlocksPerSM = 8;

struct LLOperand {
  char* ptr;
  int64_t stride;  // elements; 0 = broadcast scalar
};

template <int NIN, int NOUT>
struct LLParams {
  int64_t n;
  LLOperand in[NIN];
  LLOperand out[NOUT];
  double* partials;  // value_and_grad: one per block
};

template <typename T> struct LLMath;
template <> struct LLMath<double> {
  __device__ static double log_(double v) { return log(v); }
  __device__ static double lgamma_(double v) { return lgamma_d(v); }
  __device__ static double digamma_(double v) { return digamma_d(v); }
  __device__ static double trigamma_(double v) { return trigamma_d(v); }
};
template <> struct LLMath<float> {
  __device__ static float log_(float v) { return logf(v); }
  __device__ static float lgamma_(float v) { return lgamma_m(v); }
  __device__ static float digamma_(float v) { return digamma_m(v); }
  __device__ static float trigamma_(float v) { return trigamma_m(v); }
};

template <typename TS, typename T>
__device__ __forceinline__ T ll_load(const LLOperand& o, int64_t i) {
  return load_as<TS, T>(o.ptr + i * o.stride * (int64_t)sizeof(TS));
}

// in = {x, k, θ}; out = {L (partials), ∂/∂x, ∂/∂k, ∂/∂θ}; out[o].ptr == NULL: not requested.
template <typename TS, typename T>
__global__ void __launch_bounds__(kLLBlock) gll_value_grad_kernel(const LLParams<3, 4> p) {
  using M = LLMath<T>;
  __shared__ double s_warp[kLLBlock / 32];
  double acc = 0.0;
  const int64_t step = (int64_t)gridDim.x * kLLBlock;
  for (int64_t i = (int64_t)blockIdx.x * kLLBlock + threadIdx.x; i < p.n; i += step) {
    const T x = ll_load<TS, T>(p.in[0], i), k = ll_load<TS, T>(p.in[1], i), th = ll_load<TS, T>(p.in[2], i);
    const T lx = M::log_(x), lt = M::log_(th), rt = T(1) / th;
    const T ell = (k - T(1)) * lx - x * rt - M::lgamma_(k) - k * lt;
    acc += (double)ell;
    if (p.out[1].ptr) store_as<TS>(p.out[1].ptr + i * p.out[1].stride * (int64_t)sizeof(TS), (k - T(1)) / x - rt);
    if (p.out[2].ptr) store_as<TS>(p.out[2].ptr + i * p.out[2].stride * (int64_t)sizeof(TS), lx - M::digamma_(k) - lt);
    if (p.out[3].ptr) store_as<TS>(p.out[3].ptr + i * p.out[3].stride * (int64_t)sizeof(TS), (x * rt - k) * rt);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kLLBlock / 32; ++w) s += s_warp[w];
    p.partials[blockIdx.x] = s;
  }
}

// in = {g, x, k, θ, u_x, u_k, u_θ} (u's with ptr NULL are zero); out = g·H·u components.
template <typename TS, typename T>
__global__ void __launch_bounds__(kLLBlock) gll_hvp_kernel(const LLParams<7, 3> p) {
  using M = LLMath<T>;
  const int64_t step = (int64_t)gridDim.x * kLLBlock;
  for (int64_t i = (int64_t)blockIdx.x * kLLBlock + threadIdx.x; i < p.n; i += step) {
    const T g = ll_load<TS, T>(p.in[0], i), x = ll_load<TS, T>(p.in[1], i), k = ll_load<TS, T>(p.in[2], i),
            th = ll_load<TS, T>(p.in[3], i);
    const T ux = p.in[4].ptr ? ll_load<TS, T>(p.in[4], i) : T(0);
    const T uk = p.in[5].ptr ? ll_load<TS, T>(p.in[5], i) : T(0);
    const T ut = p.in[6].ptr ? ll_load<TS, T>(p.in[6], i) : T(0);
    const T rx = T(1) / x, rt = T(1) / th, rt2 = rt * rt;
    if (p.out[0].ptr)
      store_as<TS>(p.out[0].ptr + i * p.out[0].stride * (int64_t)sizeof(TS),
                   g * (-(k - T(1)) * rx * rx * ux + rx * uk + rt2 * ut));
    if (p.out[1].ptr)
      store_as<TS>(p.out[1].ptr + i * p.out[1].stride * (int64_t)sizeof(TS),
                   g * (rx * ux - (uk != T(0) ? M::trigamma_(k) * uk : T(0)) - rt * ut));
    if (p.out[2].ptr)
      store_as<TS>(p.out[2].ptr + i * p.out[2].stride * (int64_t)sizeof(TS),
                   g * (rt2 * ux - rt * uk + (k - T(2) * x * rt) * rt2 * ut));
  }
}

// Validates the operands (one iteration shape that coalesces to at most one
// dimension, every operand contiguous or a broadcast scalar) and fills the
// per-operand strides.
template <int NIN, int NOUT>
int32_t ll_prepare(const tsb_tensor* in, int32_t n_in, const tsb_tensor* out, int32_t n_out, bool first_out_is_sum,
                   LLParams<NIN, NOUT>& p, int32_t& dtype, int64_t& numel) {
  if (n_in != NIN || n_out != NOUT)
    return set_error(TSB_ERR_ARGUMENT, "expected %d inputs and %d outputs, got %d and %d", NIN, NOUT, n_in, n_out);
  if (!in || !out) return set_error(TSB_ERR_ARGUMENT, "null operand array");
  // the first input (x, or g for the Hessian-vector product) fixes dtype
  // and shape; its data may be NULL only for an empty shape
  const tsb_tensor& r = in[0];
  if (r.ndim < 0 || r.ndim > TSB_MAX_DIMS) return set_error(TSB_ERR_ARGUMENT, "ndim %d out of range", r.ndim);
  dtype = r.dtype;
  if (dtype_size(dtype) == 0) return set_error(TSB_ERR_DTYPE, "unknown dtype code %d", dtype);
  numel = 1;
  for (int d = 0; d < r.ndim; ++d) {
    if (r.sizes[d] < 0) return set_error(TSB_ERR_ARGUMENT, "negative size");
    numel *= r.sizes[d];
  }
  p.n = numel;
  if (numel > 0 && !r.data) return set_error(TSB_ERR_ARGUMENT, "input 0 has a null data pointer");
  // stride of a 1-D walk over the shape: every dim's stride equals the
  // contiguous stride, or every stride is zero (a broadcast scalar)
  auto walk = [&](const tsb_tensor& t, int64_t& stride) -> int32_t {
    if (t.dtype != dtype) return set_error(TSB_ERR_DTYPE, "operands have different dtypes");
    if (t.ndim != r.ndim) return set_error(TSB_ERR_ARGUMENT, "operands have different ndim");
    bool all_zero = true, contiguous = true;
    int64_t expect = 1;
    for (int d = t.ndim - 1; d >= 0; --d) {
      if (t.sizes[d] != r.sizes[d]) return set_error(TSB_ERR_ARGUMENT, "operand sizes differ from the iteration shape");
      if (t.sizes[d] == 1) continue;
      if (t.strides[d] != 0) all_zero = false;
      if (t.strides[d] != expect) contiguous = false;
      expect *= t.sizes[d];
    }
    if (((uintptr_t)t.data) % (uintptr_t)dtype_size(dtype) != 0) return set_error(TSB_ERR_ARGUMENT, "misaligned operand");
    if (numel == 0) {
      stride = 0;
      return TSB_OK;
    }
    if (all_zero) {
      stride = 0;
      return TSB_OK;
    }
    if (contiguous) {
      stride = 1;
      return TSB_OK;
    }
    return set_error(TSB_ERR_LAYOUT, "operands must be contiguous or broadcast scalars over the iteration shape");
  };
  for (int k = 0; k < NIN; ++k) {
    p.in[k].ptr = static_cast<char*>(in[k].data);
    p.in[k].stride = 0;
    if (!in[k].data && (k > 0 || numel > 0)) continue;
    const int32_t st = walk(in[k], p.in[k].stride);
    if (st) return st;
  }
  for (int o = 0; o < NOUT; ++o) {
    p.out[o].ptr = static_cast<char*>(out[o].data);
    p.out[o].stride = 0;
    if (!out[o].data) continue;
    const int32_t st = walk(out[o], p.out[o].stride);
    if (st) return st;
    if (first_out_is_sum && o == 0) {
      if (p.out[0].stride != 0 && numel > 1)
        return set_error(TSB_ERR_ARGUMENT, "the value output must be reduced (stride 0) over the iteration shape");
    } else if (p.out[o].stride == 0 && numel > 1) {
      return set_error(TSB_ERR_ARGUMENT, "per-element output %d must not be broadcast", o);
    }
  }
  return TSB_OK;
}

int ll_grid(int64_t n, const DeviceInfo* info) {
  const int64_t want = (n + kLLBlock - 1) / kLLBlock;
  const int64_t cap = (int64_t)info->sm_count * kLLBlocksPerSM;
  return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

}  // namespace
}  // namespace tsb

extern "C" int64_t tsb_gamma_log_likelihood_workspace_bytes(void) {
  int dev = 0;
  const tsb::DeviceInfo* info = nullptr;
  if (tsb::current_device(&dev, &info)) return TSB_ERR_DEVICE;
  return tsb::align256((int64_t)info->sm_count * tsb::kLLBlocksPerSM * (int64_t)sizeof(double));
}

extern "C" TSB_OP_SIGNATURE(tsb_gamma_log_likelihood_value_and_grad) {
  tsb::LLParams<3, 4> p;
  int32_t dtype = 0;
  int64_t numel = 0;
  int32_t st = tsb::ll_prepare<3, 4>(in, n_in, out, n_out, true, p, dtype, numel);
  if (st) return st;
  for (int k = 0; k < 3; ++k)
    if (numel > 0 && !in[k].data) return tsb::set_error(TSB_ERR_ARGUMENT, "input %d has a null data pointer", k);
  if (precision != TSB_PRECISION_AUTO && precision != TSB_PRECISION_FP64)
    return tsb::set_error(TSB_ERR_ARGUMENT, "unknown precision mode %d", precision);
  int dev = 0;
  const tsb::DeviceInfo* info = nullptr;
  st = tsb::current_device(&dev, &info);
  if (st) return st;
  // every launch writes one partial sum per block (unused when the value is
  // not requested); an empty input gives L = 0
  const int grid = tsb::ll_grid(numel, info);
  if (!workspace || workspace_bytes < (int64_t)grid * 8 || ((uintptr_t)workspace % 256) != 0)
    return tsb::set_error(TSB_ERR_WORKSPACE,
                          "%lld bytes of 256-byte aligned workspace needed (tsb_gamma_log_likelihood_workspace_bytes)",
                          (long long)grid * 8);
  p.partials = static_cast<double*>(workspace);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool use64 = precision == TSB_PRECISION_FP64;
  switch (dtype) {
    case TSB_F64: tsb::gll_value_grad_kernel<double, double><<<grid, tsb::kLLBlock, 0, s>>>(p); break;
    case TSB_F32:
      if (use64) tsb::gll_value_grad_kernel<float, double><<<grid, tsb::kLLBlock, 0, s>>>(p);
      else tsb::gll_value_grad_kernel<float, float><<<grid, tsb::kLLBlock, 0, s>>>(p);
      break;
    case TSB_F16: tsb::gll_value_grad_kernel<__half, float><<<grid, tsb::kLLBlock, 0, s>>>(p); break;
    case TSB_BF16: tsb::gll_value_grad_kernel<__nv_bfloat16, float><<<grid, tsb::kLLBlock, 0, s>>>(p); break;
    default: return tsb::set_error(TSB_ERR_DTYPE, "unsupported dtype");
  }
  tsb::count_launches(1);
  st = tsb::check_launch("likelihood kernel launch");
  if (st || !out[0].data) return st;
  switch (dtype) {
    case TSB_F64: tsb::finalize_all_kernel<double><<<1, tsb::kBlock, 0, s>>>(p.partials, grid, p.out[0].ptr); break;
    case TSB_F32: tsb::finalize_all_kernel<float><<<1, tsb::kBlock, 0, s>>>(p.partials, grid, p.out[0].ptr); break;
    case TSB_F16: tsb::finalize_all_kernel<__half><<<1, tsb::kBlock, 0, s>>>(p.partials, grid, p.out[0].ptr); break;
    case TSB_BF16:
      tsb::finalize_all_kernel<__nv_bfloat16><<<1, tsb::kBlock, 0, s>>>(p.partials, grid, p.out[0].ptr);
      break;
  }
  tsb::count_launches(1);
  return tsb::check_launch("likelihood finalize launch");
}

extern "C" TSB_OP_SIGNATURE(tsb_gamma_log_likelihood_hvp) {
  tsb::LLParams<7, 3> p;
  int32_t dtype = 0;
  int64_t numel = 0;
  int32_t st = tsb::ll_prepare<7, 3>(in, n_in, out, n_out, false, p, dtype, numel);
  if (st) return st;
  for (int k = 0; k < 4; ++k)
    if (numel > 0 && !in[k].data) return tsb::set_error(TSB_ERR_ARGUMENT, "input %d has a null data pointer", k);
  if (precision != TSB_PRECISION_AUTO && precision != TSB_PRECISION_FP64)
    return tsb::set_error(TSB_ERR_ARGUMENT, "unknown precision mode %d", precision);
  (void)workspace;
  (void)workspace_bytes;
  if (numel == 0) return TSB_OK;
  int dev = 0;
  const tsb::DeviceInfo* info = nullptr;
  st = tsb::current_device(&dev, &info);
  if (st) return st;
  const int grid = tsb::ll_grid(numel, info);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool use64 = precision == TSB_PRECISION_FP64;
  switch (dtype) {
    case TSB_F64: tsb::gll_hvp_kernel<double, double><<<grid, tsb::kLLBlock, 0, s>>>(p); break;
    case TSB_F32:
      if (use64) tsb::gll_hvp_kernel<float, double><<<grid, tsb::kLLBlock, 0, s>>>(p);
      else tsb::gll_hvp_kernel<float, float><<<grid, tsb::kLLBlock, 0, s>>>(p);
      break;
    case TSB_F16: tsb::gll_hvp_kernel<__half, float><<<grid, tsb::kLLBlock, 0, s>>>(p); break;
    case TSB_BF16: tsb::gll_hvp_kernel<__nv_bfloat16, float><<<grid, tsb::kLLBlock, 0, s>>>(p); break;
    default: return tsb::set_error(TSB_ERR_DTYPE, "unsupported dtype");
  }
  tsb::count_launches(1);
  return tsb::check_launch("likelihood hvp kernel launch");
}
