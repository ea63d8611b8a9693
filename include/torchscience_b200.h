/*
 * torchscience_b200 — C ABI of the sm_100a special-function kernels.
 *
 * This library replaces the per-element CPU loops of torchscience's special
 * functions (TensorIterator + at::native::cpu_kernel over the scalar templates
 * in src/torchscience/csrc/kernel/special_functions/*.h, instantiated by
 * src/torchscience/csrc/cpu/special_functions.h) with CUDA kernels.  It has no
 * torch types in its signatures: every operand is a `tsb_tensor` (a device
 * pointer plus sizes and element strides over the common iteration shape).
 *
 * Conventions shared by every entry point below:
 *   - `in` / `out` hold n_in / n_out operands, in the order of the matching
 *     torchscience schema (src/torchscience/csrc/torchscience.cpp), e.g. for
 *     regularized_gamma_p_backward: in = {grad, a, x}, out = {grad_a, grad_x}.
 *   - all operands share `ndim` and `sizes` (the broadcast iteration shape);
 *     an input broadcast along a dim has stride 0 there.
 *   - an OUTPUT with stride 0 along a dim of size > 1 is a reduced output: the
 *     kernel sums the per-element values over that dim (deterministically, in
 *     double, in a fixed order).  This is how backward kernels return
 *     gradients already reduced to an input's shape.  Reduced outputs need a
 *     device workspace of tsb_workspace_bytes(...) bytes.
 *   - a grid of an (R, 1) input against a (1, C) input (or the transpose)
 *     also asks for a small workspace (tsb_workspace_bytes > 0 even with no
 *     reduced output): the incomplete-gamma entry points use it to evaluate
 *     the grid in rows sorted by the shape parameter (one warp per 32 sorted
 *     rows), which keeps the lanes of a warp on the same code path.  Without
 *     it (workspace NULL or too small, no reduced output) they run the
 *     unsorted tile kernel and give the same values.
 *   - an output whose `data` is NULL is not requested and is not computed.
 *   - all operands of one call have the same dtype.
 *   - precision: TSB_PRECISION_AUTO picks the FP64 kernels for f64 data and
 *     the mixed FP32 kernels (FP32 bulk, FP64 only in the classified bins that
 *     need it) for f32/f16/bf16 data; TSB_PRECISION_FP64 runs the FP64
 *     kernels for any dtype.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  Calls are
 *     asynchronous and stream-ordered; the library keeps no per-call state.
 *   - return value: TSB_OK or a negative tsb_status; tsb_last_error() gives a
 *     message for the calling thread.  Nothing is launched on error.
 */
#ifndef TORCHSCIENCE_B200_H_
#define TORCHSCIENCE_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TSB_MAX_DIMS 8

typedef enum tsb_dtype {
  TSB_F32 = 0,
  TSB_F64 = 1,
  TSB_F16 = 2,
  TSB_BF16 = 3,
  TSB_C64 = 4,   /* complex64: interleaved float real, imaginary */
  TSB_C128 = 5   /* complex128: interleaved double real, imaginary */
} tsb_dtype;

typedef enum tsb_precision {
  TSB_PRECISION_AUTO = 0,
  TSB_PRECISION_FP64 = 1
} tsb_precision;

typedef enum tsb_status {
  TSB_OK = 0,
  TSB_ERR_ARGUMENT = -1,    /* null pointer, bad count, bad ndim/sizes */
  TSB_ERR_DTYPE = -2,       /* unknown or mixed dtypes */
  TSB_ERR_LAYOUT = -3,      /* reduced-output pattern this kernel cannot fuse */
  TSB_ERR_WORKSPACE = -4,   /* workspace missing or too small */
  TSB_ERR_LAUNCH = -5,      /* CUDA launch error */
  TSB_ERR_DEVICE = -6       /* no usable sm_100 device */
} tsb_status;

typedef struct tsb_tensor {
  void* data;                      /* device pointer to element [0,...,0] */
  int32_t dtype;                   /* tsb_dtype */
  int32_t ndim;                    /* 0 .. TSB_MAX_DIMS */
  int64_t sizes[TSB_MAX_DIMS];     /* iteration shape */
  int64_t strides[TSB_MAX_DIMS];   /* element strides (0 = broadcast/reduced) */
} tsb_tensor;

/* Library / error helpers. */
const char* tsb_version(void);
const char* tsb_last_error(void);
const char* tsb_status_string(int32_t status);

/* Bytes of device workspace (256-byte aligned) that an entry point called with
 * these operands needs: 0 when no output is reduced, negative (a tsb_status)
 * when the operands are invalid.  The reference has no counterpart: its CPU
 * backward writes full-shape gradients and lets the autograd engine reduce
 * them (cpu/macros.h:987-1032). */
int64_t tsb_workspace_bytes(const tsb_tensor* in, int32_t n_in, const tsb_tensor* out, int32_t n_out);

/* Number of CUDA kernels this library has launched in this process, over all
 * devices and threads (a diagnostic for counting launches; no counterpart in
 * the reference, whose operators run on the CPU). */
int64_t tsb_launch_count(void);

/* Number of elements, since the last reset, whose series, continued fraction
 * or recurrence stopped at its iteration cap on the current device (their
 * results are truncated sums: every loop is bounded, so such inputs cost
 * time, never a hang).  Waits for the device to finish its work first.
 * reset != 0 zeroes the counters after reading them.  Negative: a
 * tsb_status.  The reference stops its loops at fixed caps too
 * (regularized_gamma_p.h:12,30: max_iter = 200) without reporting it. */
int64_t tsb_unconverged_count(int32_t reset);

/* Every op entry point has this signature. */
#define TSB_OP_SIGNATURE(name)                                               \
  int32_t name(const tsb_tensor* in, int32_t n_in, const tsb_tensor* out,    \
               int32_t n_out, int32_t precision, void* workspace,            \
               int64_t workspace_bytes, void* stream)

/* ---- Gamma family ------------------------------------------------------ */
/* log_gamma(z): replaces kernel/special_functions/log_gamma.h:23-65, schema
 * torchscience.cpp:849; backward log_gamma_backward.h:8-10 (:850),
 * backward_backward log_gamma_backward_backward.h:11-20 (:851). */
TSB_OP_SIGNATURE(tsb_log_gamma);
TSB_OP_SIGNATURE(tsb_log_gamma_backward);
TSB_OP_SIGNATURE(tsb_log_gamma_backward_backward);
/* gamma(z): gamma.h:68-122, schema torchscience.cpp:813-815. */
TSB_OP_SIGNATURE(tsb_gamma);
TSB_OP_SIGNATURE(tsb_gamma_backward);
TSB_OP_SIGNATURE(tsb_gamma_backward_backward);
/* digamma(z): digamma.h:10-25, schema torchscience.cpp:817-819. */
TSB_OP_SIGNATURE(tsb_digamma);
TSB_OP_SIGNATURE(tsb_digamma_backward);
TSB_OP_SIGNATURE(tsb_digamma_backward_backward);
/* trigamma(z): trigamma.h:10-25 (+ tetragamma.h:11-30 in its backward),
 * schema torchscience.cpp:821-823. */
TSB_OP_SIGNATURE(tsb_trigamma);
TSB_OP_SIGNATURE(tsb_trigamma_backward);
TSB_OP_SIGNATURE(tsb_trigamma_backward_backward);
/* polygamma(n, z), order truncated toward zero, NaN for n <= -1: polygamma.h:45-62, schema
 * torchscience.cpp:841-843; backward polygamma_backward.h:10-19 (outputs grad_n = 0,
 * grad_z = grad·ψ^(n+1)(z)); double backward polygamma_backward_backward.h:10-22. */
TSB_OP_SIGNATURE(tsb_polygamma);
TSB_OP_SIGNATURE(tsb_polygamma_backward);
TSB_OP_SIGNATURE(tsb_polygamma_backward_backward);
/* log_beta(a, b) = ln|B(a, b)|: log_beta.h:10-13, schema torchscience.cpp:845-847; backward
 * log_beta_backward.h:10-17; double backward log_beta_backward_backward.h:10-33. */
TSB_OP_SIGNATURE(tsb_log_beta);
TSB_OP_SIGNATURE(tsb_log_beta_backward);
TSB_OP_SIGNATURE(tsb_log_beta_backward_backward);
/* beta(a, b): beta.h:12-15, schema torchscience.cpp:825-827; backward beta_backward.h:13-27;
 * double backward beta_backward_backward.h:10-30.  Signed for negative arguments. */
TSB_OP_SIGNATURE(tsb_beta);
TSB_OP_SIGNATURE(tsb_beta_backward);
TSB_OP_SIGNATURE(tsb_beta_backward_backward);

/* ---- Regularized incomplete gamma ------------------------------------- */
/* regularized_gamma_p(a, x): regularized_gamma_p.h:57-71, schema
 * torchscience.cpp:853-855; backward regularized_gamma_p_backward.h:27-33,
 * backward_backward regularized_gamma_p_backward_backward.h:12-41. */
TSB_OP_SIGNATURE(tsb_regularized_gamma_p);
TSB_OP_SIGNATURE(tsb_regularized_gamma_p_backward);
TSB_OP_SIGNATURE(tsb_regularized_gamma_p_backward_backward);
/* regularized_gamma_q(a, x): regularized_gamma_q.h:13-22, schema
 * torchscience.cpp:857-859; backward regularized_gamma_q_backward.h:12-16,
 * backward_backward regularized_gamma_q_backward_backward.h:12-22. */
TSB_OP_SIGNATURE(tsb_regularized_gamma_q);
TSB_OP_SIGNATURE(tsb_regularized_gamma_q_backward);
TSB_OP_SIGNATURE(tsb_regularized_gamma_q_backward_backward);

/* Allocation-free regularized_gamma_p backward (no counterpart in the
 * reference, whose CPU backward leaves the reduction of broadcast gradients
 * to the autograd engine).  Same operands and results as
 * tsb_regularized_gamma_p_backward, but it takes no workspace: for callers
 * that cannot allocate device memory (hosts reaching this library only
 * through a C FFI, with no device allocator of their own; loops that must not
 * call cudaMalloc, which can synchronize the device).  The partial sums of
 * reduced gradients go to a fixed file-scope device array of
 * TSB_NOALLOC_SCRATCH_BYTES that each GPU loading the library keeps until
 * exit; requests needing more return TSB_ERR_WORKSPACE without launching.
 * The first call on a device looks up the array's address and should come
 * before any stream capture.  The address is cached per device for the life
 * of the process: after cudaDeviceReset (which unloads this library's device
 * code with the context) the entry point must not be called again in that
 * process.  All calls share the array: calls that overlap on the GPU race
 * and must be serialized by the caller. */
#define TSB_NOALLOC_SCRATCH_BYTES (8ll << 20)
int32_t tsb_regularized_gamma_p_backward_noalloc(const tsb_tensor* in, int32_t n_in, const tsb_tensor* out,
                                                 int32_t n_out, int32_t precision, void* stream);

/* ---- Fused Gamma log-likelihood ------------------------------------------ */
/* No single counterpart in the reference: its Gamma log-likelihood is a chain
 * of ops around log_gamma (log_gamma.h:23-65; gradient via digamma as in
 * kernel/probability/gamma_probability_density_backward.h:11-31; second
 * derivatives via trigamma as in log_gamma_backward_backward.h:11-20).  Per
 * element l = (k-1) ln x - x/theta - lnGamma(k) - k ln theta for x ~ Gamma(k, theta).
 *
 * tsb_gamma_log_likelihood_value_and_grad: in = {x, k, theta}; out = {L,
 * dL/dx, dL/dk, dL/dtheta}.  L is the sum over the iteration shape (its
 * descriptor has stride 0 in every dim), added in double in a fixed order;
 * the gradients are per element; any output may be NULL.  One pass over the
 * inputs.  Operands must be contiguous or broadcast scalars over the shape
 * (TSB_ERR_LAYOUT otherwise).  Needs tsb_gamma_log_likelihood_workspace_bytes()
 * bytes of workspace on the current device. */
int64_t tsb_gamma_log_likelihood_workspace_bytes(void);
TSB_OP_SIGNATURE(tsb_gamma_log_likelihood_value_and_grad);
/* tsb_gamma_log_likelihood_hvp: in = {g, x, k, theta, u_x, u_k, u_theta}; out =
 * the three components of g * H u per element, H the per-element Hessian of l
 * in (x, k, theta).  Any u may be NULL (zero); any output may be NULL. */
TSB_OP_SIGNATURE(tsb_gamma_log_likelihood_hvp);

/* ---- Bessel functions --------------------------------------------------- */
/* bessel_j_0(z): bessel_j_0.h:91-129, schema torchscience.cpp:872-874;
 * backward bessel_j_0_backward.h:27-30, backward_backward bessel_j_0_backward_backward.h:16-30. */
TSB_OP_SIGNATURE(tsb_bessel_j_0);
TSB_OP_SIGNATURE(tsb_bessel_j_0_backward);
TSB_OP_SIGNATURE(tsb_bessel_j_0_backward_backward);
/* Integer orders 0 and 1 as unary ops; double backward gives {gg·f'(z), gg·grad·f''(z)}. */
/* bessel_j_1(z): bessel_j_1.h:93-117, schema torchscience.cpp:877-879; J1 (odd); backward J0 - J1/z (1/2 at 0). */
TSB_OP_SIGNATURE(tsb_bessel_j_1);
TSB_OP_SIGNATURE(tsb_bessel_j_1_backward);
TSB_OP_SIGNATURE(tsb_bessel_j_1_backward_backward);
/* bessel_y_0(z): bessel_y_0.h:95-116, schema torchscience.cpp:882-884; Y0: NaN for z < 0, -inf at 0; backward -Y1 (NaN for z <= 0). */
TSB_OP_SIGNATURE(tsb_bessel_y_0);
TSB_OP_SIGNATURE(tsb_bessel_y_0_backward);
TSB_OP_SIGNATURE(tsb_bessel_y_0_backward_backward);
/* bessel_y_1(z): bessel_y_1.h:94-116, schema torchscience.cpp:887-889; Y1: NaN for z < 0, -inf at 0; backward Y0 - Y1/z (NaN for z <= 0). */
TSB_OP_SIGNATURE(tsb_bessel_y_1);
TSB_OP_SIGNATURE(tsb_bessel_y_1_backward);
TSB_OP_SIGNATURE(tsb_bessel_y_1_backward_backward);
/* modified_bessel_i_0(z): modified_bessel_i_0.h:71-86, schema torchscience.cpp:862-864; I0 (even); backward I1. */
TSB_OP_SIGNATURE(tsb_modified_bessel_i_0);
TSB_OP_SIGNATURE(tsb_modified_bessel_i_0_backward);
TSB_OP_SIGNATURE(tsb_modified_bessel_i_0_backward_backward);
/* modified_bessel_i_1(z): modified_bessel_i_1.h:55-74, schema torchscience.cpp:867-869; I1 (odd); backward I0 - I1/z (1/2 at 0). */
TSB_OP_SIGNATURE(tsb_modified_bessel_i_1);
TSB_OP_SIGNATURE(tsb_modified_bessel_i_1_backward);
TSB_OP_SIGNATURE(tsb_modified_bessel_i_1_backward_backward);
/* modified_bessel_k_0(z): modified_bessel_k_0.h:50-76, schema torchscience.cpp:892-894; K0: NaN for z < 0, +inf at 0; backward -K1 (NaN for z <= 0). */
TSB_OP_SIGNATURE(tsb_modified_bessel_k_0);
TSB_OP_SIGNATURE(tsb_modified_bessel_k_0_backward);
TSB_OP_SIGNATURE(tsb_modified_bessel_k_0_backward_backward);
/* modified_bessel_k_1(z): modified_bessel_k_1.h:51-78, schema torchscience.cpp:897-899; K1: NaN for z < 0, +inf at 0; backward -K0 - K1/z (NaN for z <= 0). */
TSB_OP_SIGNATURE(tsb_modified_bessel_k_1);
TSB_OP_SIGNATURE(tsb_modified_bessel_k_1_backward);
TSB_OP_SIGNATURE(tsb_modified_bessel_k_1_backward_backward);
/* bessel_j(n, z): bessel_j.h:240-316, schema torchscience.cpp:902-904;
 * backward bessel_j_backward.h:51-63 (grad_n, grad_z), backward_backward bessel_j_backward_backward.h. */
TSB_OP_SIGNATURE(tsb_bessel_j);
TSB_OP_SIGNATURE(tsb_bessel_j_backward);
TSB_OP_SIGNATURE(tsb_bessel_j_backward_backward);
/* bessel_y(n, z): bessel_y.h:131-193, schema torchscience.cpp:907-909;
 * backward bessel_y_backward.h:51, backward_backward bessel_y_backward_backward.h. */
TSB_OP_SIGNATURE(tsb_bessel_y);
TSB_OP_SIGNATURE(tsb_bessel_y_backward);
TSB_OP_SIGNATURE(tsb_bessel_y_backward_backward);
/* modified_bessel_i(n, z): modified_bessel_i.h:271-366, schema torchscience.cpp:917-919;
 * backward modified_bessel_i_backward.h:51, backward_backward modified_bessel_i_backward_backward.h. */
TSB_OP_SIGNATURE(tsb_modified_bessel_i);
TSB_OP_SIGNATURE(tsb_modified_bessel_i_backward);
TSB_OP_SIGNATURE(tsb_modified_bessel_i_backward_backward);
/* modified_bessel_k(n, z): modified_bessel_k.h:249-307, schema torchscience.cpp:912-914;
 * backward modified_bessel_k_backward.h:51, backward_backward modified_bessel_k_backward_backward.h. */
TSB_OP_SIGNATURE(tsb_modified_bessel_k);
TSB_OP_SIGNATURE(tsb_modified_bessel_k_backward);
TSB_OP_SIGNATURE(tsb_modified_bessel_k_backward_backward);

/* ---- Gauss hypergeometric function ----------------------------------- */
/* hypergeometric_2_f_1(a, b, c, z) for real arguments: hypergeometric_2_f_1.h:203-295,
 * schema torchscience.cpp:837-839; backward hypergeometric_2_f_1_backward.h:60-118
 * (outputs grad_a, grad_b, grad_c, grad_z), backward_backward
 * hypergeometric_2_f_1_backward_backward.h:12-125 (inputs gg_a, gg_b, gg_c, gg_z,
 * grad_output, a, b, c, z; outputs gg_out, grad_a, grad_b, grad_c, grad_z).
 * Every precision mode evaluates in FP64. */
TSB_OP_SIGNATURE(tsb_hypergeometric_2_f_1);
TSB_OP_SIGNATURE(tsb_hypergeometric_2_f_1_backward);
TSB_OP_SIGNATURE(tsb_hypergeometric_2_f_1_backward_backward);

/* ---- Spherical Bessel functions of order 0 and 1 (unary) ------------------ */
/* spherical_bessel_j_0(z): kernel/special_functions/spherical_bessel_j_0.h:33-44, schema torchscience.cpp:922-924. */
TSB_OP_SIGNATURE(tsb_spherical_bessel_j_0);
TSB_OP_SIGNATURE(tsb_spherical_bessel_j_0_backward);
TSB_OP_SIGNATURE(tsb_spherical_bessel_j_0_backward_backward);
/* spherical_bessel_j_1(z): kernel/special_functions/spherical_bessel_j_1.h:33-45, schema torchscience.cpp:927-929. */
TSB_OP_SIGNATURE(tsb_spherical_bessel_j_1);
TSB_OP_SIGNATURE(tsb_spherical_bessel_j_1_backward);
TSB_OP_SIGNATURE(tsb_spherical_bessel_j_1_backward_backward);
/* spherical_bessel_y_0(z): kernel/special_functions/spherical_bessel_y_0.h:33-41, schema torchscience.cpp:937-939. */
TSB_OP_SIGNATURE(tsb_spherical_bessel_y_0);
TSB_OP_SIGNATURE(tsb_spherical_bessel_y_0_backward);
TSB_OP_SIGNATURE(tsb_spherical_bessel_y_0_backward_backward);
/* spherical_bessel_y_1(z): kernel/special_functions/spherical_bessel_y_1.h:33-42, schema torchscience.cpp:942-944. */
TSB_OP_SIGNATURE(tsb_spherical_bessel_y_1);
TSB_OP_SIGNATURE(tsb_spherical_bessel_y_1_backward);
TSB_OP_SIGNATURE(tsb_spherical_bessel_y_1_backward_backward);
/* spherical_bessel_i_0(z): kernel/special_functions/spherical_bessel_i_0.h:33-47, schema torchscience.cpp:952-954. */
TSB_OP_SIGNATURE(tsb_spherical_bessel_i_0);
TSB_OP_SIGNATURE(tsb_spherical_bessel_i_0_backward);
TSB_OP_SIGNATURE(tsb_spherical_bessel_i_0_backward_backward);
/* spherical_bessel_i_1(z): kernel/special_functions/spherical_bessel_i_1.h:33-45, schema torchscience.cpp:957-959. */
TSB_OP_SIGNATURE(tsb_spherical_bessel_i_1);
TSB_OP_SIGNATURE(tsb_spherical_bessel_i_1_backward);
TSB_OP_SIGNATURE(tsb_spherical_bessel_i_1_backward_backward);
/* spherical_bessel_k_0(z): kernel/special_functions/spherical_bessel_k_0.h:33-49, schema torchscience.cpp:967-969. */
TSB_OP_SIGNATURE(tsb_spherical_bessel_k_0);
TSB_OP_SIGNATURE(tsb_spherical_bessel_k_0_backward);
TSB_OP_SIGNATURE(tsb_spherical_bessel_k_0_backward_backward);
/* spherical_bessel_k_1(z): kernel/special_functions/spherical_bessel_k_1.h:33-46, schema torchscience.cpp:972-974. */
TSB_OP_SIGNATURE(tsb_spherical_bessel_k_1);
TSB_OP_SIGNATURE(tsb_spherical_bessel_k_1_backward);
TSB_OP_SIGNATURE(tsb_spherical_bessel_k_1_backward_backward);

/* ---- Spherical Bessel functions of real order (n, z) ----------------------- */
/* f_n(z) = sqrt(pi/(2|z|)) C_{n+1/2}(|z|), C = J, Y, I, K, with the reference's conventions for z < 0 and
 * |z| < 1e-12; backward outputs {grad_n (central difference in n), grad_z}. */
/* spherical_bessel_j(n, z): kernel/special_functions/spherical_bessel_j.h, schema torchscience.cpp:932-934. */
TSB_OP_SIGNATURE(tsb_spherical_bessel_j);
TSB_OP_SIGNATURE(tsb_spherical_bessel_j_backward);
TSB_OP_SIGNATURE(tsb_spherical_bessel_j_backward_backward);
/* spherical_bessel_y(n, z): kernel/special_functions/spherical_bessel_y.h, schema torchscience.cpp:947-949. */
TSB_OP_SIGNATURE(tsb_spherical_bessel_y);
TSB_OP_SIGNATURE(tsb_spherical_bessel_y_backward);
TSB_OP_SIGNATURE(tsb_spherical_bessel_y_backward_backward);
/* spherical_bessel_i(n, z): kernel/special_functions/spherical_bessel_i.h, schema torchscience.cpp:962-964. */
TSB_OP_SIGNATURE(tsb_spherical_bessel_i);
TSB_OP_SIGNATURE(tsb_spherical_bessel_i_backward);
TSB_OP_SIGNATURE(tsb_spherical_bessel_i_backward_backward);
/* spherical_bessel_k(n, z): kernel/special_functions/spherical_bessel_k.h, schema torchscience.cpp:977-979. */
TSB_OP_SIGNATURE(tsb_spherical_bessel_k);
TSB_OP_SIGNATURE(tsb_spherical_bessel_k_backward);
TSB_OP_SIGNATURE(tsb_spherical_bessel_k_backward_backward);

/* ---- Regularized incomplete beta I_x(a, b) --------------------------------- */
/* incomplete_beta(x, a, b): kernel/special_functions/incomplete_beta.h:27-63, schema torchscience.cpp:833-835;
 * backward incomplete_beta_backward.h:212-276 (outputs {grad_x, grad_a, grad_b}); double backward
 * incomplete_beta_backward_backward.h:110-237 (outputs {grad_grad_output, grad_x, grad_a, grad_b}). */
TSB_OP_SIGNATURE(tsb_incomplete_beta);
TSB_OP_SIGNATURE(tsb_incomplete_beta_backward);
TSB_OP_SIGNATURE(tsb_incomplete_beta_backward_backward);

/* ---- Fused forward for autograd (no counterpart in the reference) -------- */
/* regularized_gamma_p / _q with their first derivatives in one evaluation: in = {a, x}, out =
 * {P (Q), d/da, d/dx} at the broadcast shape; a NULL d/da output is skipped.  The autograd forward of
 * regularized_gamma_p/_q uses it when an input requires grad and keeps the derivatives, so the backward
 * is tsb_gradient_product instead of a second evaluation (the reference's autograd calls
 * regularized_gamma_p and later regularized_gamma_p_backward, autograd/special_functions.h:15). */
TSB_OP_SIGNATURE(tsb_regularized_gamma_p_forward_with_grads);
TSB_OP_SIGNATURE(tsb_regularized_gamma_q_forward_with_grads);
/* in = {grad, d_a, d_b}, out = {grad*d_a, grad*d_b}, each reduced (summed) to its output's shape when
 * that output broadcasts, like the reduced backward entry points. */
TSB_OP_SIGNATURE(tsb_gradient_product);

/* ---- Probability callers of the incomplete gamma ----------------------- */
/* gamma_cumulative_distribution(x, shape, scale): kernel/probability/gamma_cumulative_distribution.h:9-13,
 * schema torchscience.cpp:1909-1910; backward gamma_cumulative_distribution_backward.h:16-43
 * (outputs grad_x, grad_shape, grad_scale). */
TSB_OP_SIGNATURE(tsb_gamma_cumulative_distribution);
TSB_OP_SIGNATURE(tsb_gamma_cumulative_distribution_backward);
/* chi2_cumulative_distribution(x, df): chi2_cumulative_distribution.h:9-13, schema
 * torchscience.cpp:1881-1882; backward chi2_cumulative_distribution_backward.h:31-37. */
TSB_OP_SIGNATURE(tsb_chi2_cumulative_distribution);
TSB_OP_SIGNATURE(tsb_chi2_cumulative_distribution_backward);
/* poisson_cumulative_distribution(k, rate): poisson_cumulative_distribution.h:10-18, schema
 * torchscience.cpp:1923-1924; backward poisson_cumulative_distribution_backward.h:13-29 (grad_k = 0). */
TSB_OP_SIGNATURE(tsb_poisson_cumulative_distribution);
TSB_OP_SIGNATURE(tsb_poisson_cumulative_distribution_backward);
/* chi2_survival(x, df) = Q(df/2, x/2), 1 for x <= 0: kernel/probability/chi2_survival.h:9-13, schema
 * torchscience.cpp:1887-1888; backward chi2_survival_backward.h:11-17 (the negated CDF gradients). */
TSB_OP_SIGNATURE(tsb_chi2_survival);
TSB_OP_SIGNATURE(tsb_chi2_survival_backward);
/* gamma_probability_density(x, shape, scale): gamma_probability_density.h:9-16, schema
 * torchscience.cpp:1911-1912; backward gamma_probability_density_backward.h:17-40
 * (outputs grad_x, grad_shape, grad_scale; 0 for x <= 0). */
TSB_OP_SIGNATURE(tsb_gamma_probability_density);
TSB_OP_SIGNATURE(tsb_gamma_probability_density_backward);
/* chi2_probability_density(x, df): chi2_probability_density.h:10-21 (x = 0: inf for df < 2, 1/2 for
 * df = 2, else 0), schema torchscience.cpp:1883-1884; backward chi2_probability_density_backward.h:11-40
 * (outputs grad_x, grad_df; 0 for x <= 0). */
TSB_OP_SIGNATURE(tsb_chi2_probability_density);
TSB_OP_SIGNATURE(tsb_chi2_probability_density_backward);

/* ---- Complete elliptic integrals --------------------------------------- */
/* complete_legendre_elliptic_integral_k(m): complete_legendre_elliptic_integral_k.h:29-33,
 * schema torchscience.cpp:1015-1017; backward ..._k_backward.h:24-53,
 * backward_backward ..._k_backward_backward.h:13-126. */
TSB_OP_SIGNATURE(tsb_complete_legendre_elliptic_integral_k);
TSB_OP_SIGNATURE(tsb_complete_legendre_elliptic_integral_k_backward);
TSB_OP_SIGNATURE(tsb_complete_legendre_elliptic_integral_k_backward_backward);
/* complete_legendre_elliptic_integral_e(m): complete_legendre_elliptic_integral_e.h:28-36,
 * schema torchscience.cpp:1019-1021; backward ..._e_backward.h:41-52,
 * backward_backward ..._e_backward_backward.h:17-43. */
TSB_OP_SIGNATURE(tsb_complete_legendre_elliptic_integral_e);
TSB_OP_SIGNATURE(tsb_complete_legendre_elliptic_integral_e_backward);
TSB_OP_SIGNATURE(tsb_complete_legendre_elliptic_integral_e_backward_backward);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif  /* TORCHSCIENCE_B200_H_ */
