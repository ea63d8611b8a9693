// torch.ops.torchscience.* registration for the B200 kernels.
//
// The schema strings are the reference's own (src/torchscience/csrc/torchscience.cpp,
// cited per op below) so that torch.ops.torchscience.<op>, <op>_backward and
// <op>_backward_backward keep their names, argument names and return arity.
// Implementations are registered for CUDA (the sm_100a kernels through the C
// ABI), Meta (shape/dtype via TensorIterator, as meta/macros.h:9-411 does),
// Autograd (the same Function pair structure as autograd/macros.h:5-837),
// AutocastCUDA (cast to float32 like autocast/macros.h:6-172) and CPU (an
// error: there is no CPU fallback).
#include <ATen/autocast_mode.h>
#include <torch/autograd.h>
#include <torch/library.h>

#include "pointwise.h"
#include "schemas.h"

using torch::autograd::AutogradContext;
using torch::autograd::variable_list;

namespace tsbh {

// Whether autograd's forward of regularized_gamma_p / _q keeps the first
// derivatives (one evaluation; 16 bytes per element of float64 output stay
// alive until the backward) or the backward evaluates them again from the
// inputs (no extra memory).  Process-wide; on by default.
inline std::atomic<bool>& keep_derivatives() {
  static std::atomic<bool> keep{true};
  return keep;
}

inline bool wants_grad(const at::Tensor& t) {
  return t.requires_grad() && (at::isFloatingType(t.scalar_type()) || at::isComplexType(t.scalar_type()));
}

inline bool any_cuda(std::initializer_list<at::Tensor> ts) {
  for (const auto& t : ts)
    if (t.defined() && t.is_cuda()) return true;
  return false;
}

// Tensors of a trace (torch.compile / export: fake or functional tensors)
// carry no data, so the autograd code must not call the C ABI on them: their
// kernels go through the dispatcher, which routes them to the Meta kernels.
inline bool any_traced(std::initializer_list<at::Tensor> ts) {
  for (const auto& t : ts)
    if (t.defined() && (t.is_meta() || t.key_set().has(c10::DispatchKey::Python) ||
                        t.key_set().has(c10::DispatchKey::Functionalize)))
      return true;
  return false;
}

// An autograd Function cannot return undefined tensors: gradients that were
// not requested (and so not computed) come back as a zero expanded to the
// input's shape, which allocates one element.
inline torch::autograd::variable_list defined_or_zero(std::vector<at::Tensor> r, at::TensorList like) {
  for (size_t i = 0; i < r.size(); ++i)
    if (!r[i].defined()) r[i] = at::zeros({}, like[i].options()).expand(like[i].sizes());
  return r;
}

}  // namespace tsbh

// ---------------------------------------------------------------- unary ops
// Name: op name; Cls: autograd class prefix; A: argument name in the schema.
#define TSBH_UNARY_OP(name, Cls, A, FWD, BWD, BB)                                                       \
  namespace tsbh::ops {                                                                                 \
  at::Tensor name##_cuda(const at::Tensor& a) { return run_pointwise(FWD, #name, {a}, 1)[0]; }         \
  at::Tensor name##_backward_cuda(const at::Tensor& g, const at::Tensor& a) {                          \
    return run_pointwise(BWD, #name "_backward", {g, a}, 1)[0];                                        \
  }                                                                                                     \
  std::tuple<at::Tensor, at::Tensor> name##_backward_backward_cuda(const at::Tensor& gg, const at::Tensor& g, \
                                                                    const at::Tensor& a) {            \
    if (!gg.defined()) return {};                                                                      \
    auto r = run_pointwise(BB, #name "_backward_backward", {gg, g, a}, 2);                             \
    return {r[0], r[1]};                                                                               \
  }                                                                                                     \
  at::Tensor name##_meta(const at::Tensor& a) { return meta_pointwise(#name, {a}, 1)[0]; }             \
  at::Tensor name##_backward_meta(const at::Tensor& g, const at::Tensor& a) {                          \
    return meta_pointwise(#name "_backward", {g, a}, 1)[0];                                            \
  }                                                                                                     \
  std::tuple<at::Tensor, at::Tensor> name##_backward_backward_meta(const at::Tensor& gg, const at::Tensor& g, \
                                                                    const at::Tensor& a) {            \
    if (!gg.defined()) return {};                                                                      \
    auto r = meta_pointwise(#name "_backward_backward", {gg, g, a}, 2);                                \
    return {r[0], r[1]};                                                                               \
  }                                                                                                     \
  at::Tensor name##_cpu(const at::Tensor&) { cpu_not_supported(#name); }                               \
  at::Tensor name##_backward_cpu(const at::Tensor&, const at::Tensor&) { cpu_not_supported(#name "_backward"); } \
  std::tuple<at::Tensor, at::Tensor> name##_backward_backward_cpu(const at::Tensor&, const at::Tensor&,      \
                                                                   const at::Tensor&) {               \
    cpu_not_supported(#name "_backward_backward");                                                     \
  }                                                                                                     \
  class Cls##Backward : public torch::autograd::Function<Cls##Backward> {                              \
   public:                                                                                              \
    static variable_list forward(AutogradContext* ctx, const at::Tensor& g, const at::Tensor& a, bool req) { \
      ctx->save_for_backward({g, a});                                                                  \
      ctx->saved_data["req"] = req;                                                                    \
      at::AutoDispatchBelowAutograd guard;                                                             \
      static auto op = c10::Dispatcher::singleton()                                                    \
                           .findSchemaOrThrow("torchscience::" #name "_backward", "")                  \
                           .typed<at::Tensor(const at::Tensor&, const at::Tensor&)>();                 \
      return {op.call(g, a)};                                                                          \
    }                                                                                                   \
    static variable_list backward(AutogradContext* ctx, const variable_list& go) {                     \
      auto saved = ctx->get_saved_variables();                                                          \
      const bool req = ctx->saved_data["req"].toBool();                                                \
      if (!go[0].defined() || !req) return {at::Tensor(), at::Tensor(), at::Tensor()};                 \
      at::AutoDispatchBelowAutograd guard;                                                             \
      static auto op = c10::Dispatcher::singleton()                                                    \
                           .findSchemaOrThrow("torchscience::" #name "_backward_backward", "")         \
                           .typed<std::tuple<at::Tensor, at::Tensor>(const at::Tensor&, const at::Tensor&, \
                                                                     const at::Tensor&)>();           \
      auto [gg_out, g_a] = op.call(go[0], saved[0], saved[1]);                                         \
      return {gg_out, g_a, at::Tensor()};                                                              \
    }                                                                                                   \
  };                                                                                                    \
  class Cls : public torch::autograd::Function<Cls> {                                                  \
   public:                                                                                              \
    static at::Tensor forward(AutogradContext* ctx, const at::Tensor& a) {                             \
      ctx->save_for_backward({a});                                                                     \
      ctx->saved_data["req"] = wants_grad(a);                                                          \
      at::AutoDispatchBelowAutograd guard;                                                             \
      static auto op = c10::Dispatcher::singleton()                                                    \
                           .findSchemaOrThrow("torchscience::" #name, "")                              \
                           .typed<at::Tensor(const at::Tensor&)>();                                    \
      return op.call(a);                                                                               \
    }                                                                                                   \
    static variable_list backward(AutogradContext* ctx, const variable_list& go) {                     \
      auto saved = ctx->get_saved_variables();                                                          \
      const bool req = ctx->saved_data["req"].toBool();                                                \
      auto g = Cls##Backward::apply(go[0], saved[0], req);                                             \
      return {req ? g[0] : at::Tensor()};                                                              \
    }                                                                                                   \
  };                                                                                                    \
  at::Tensor name##_autograd(const at::Tensor& a) { return Cls::apply(a); }                            \
  at::Tensor name##_autocast(const at::Tensor& a) {                                                    \
    c10::impl::ExcludeDispatchKeyGuard no_autocast(c10::DispatchKey::AutocastCUDA);                    \
    static auto op = c10::Dispatcher::singleton()                                                      \
                         .findSchemaOrThrow("torchscience::" #name, "")                                \
                         .typed<at::Tensor(const at::Tensor&)>();                                      \
    return op.call(at::autocast::cached_cast(at::kFloat, a, c10::DeviceType::CUDA));                   \
  }                                                                                                     \
  } /* namespace tsbh::ops */                                                                           \
  TORCH_LIBRARY_IMPL(torchscience, CUDA, m) {                                                           \
    m.impl(#name, tsbh::ops::name##_cuda);                                                              \
    m.impl(#name "_backward", tsbh::ops::name##_backward_cuda);                                         \
    m.impl(#name "_backward_backward", tsbh::ops::name##_backward_backward_cuda);                       \
  }                                                                                                     \
  TORCH_LIBRARY_IMPL(torchscience, Meta, m) {                                                           \
    m.impl(#name, tsbh::ops::name##_meta);                                                              \
    m.impl(#name "_backward", tsbh::ops::name##_backward_meta);                                         \
    m.impl(#name "_backward_backward", tsbh::ops::name##_backward_backward_meta);                       \
  }                                                                                                     \
  TORCH_LIBRARY_IMPL(torchscience, CPU, m) {                                                            \
    m.impl(#name, tsbh::ops::name##_cpu);                                                               \
    m.impl(#name "_backward", tsbh::ops::name##_backward_cpu);                                          \
    m.impl(#name "_backward_backward", tsbh::ops::name##_backward_backward_cpu);                        \
  }                                                                                                     \
  TORCH_LIBRARY_IMPL(torchscience, Autograd, m) { m.impl(#name, tsbh::ops::name##_autograd); }         \
  TORCH_LIBRARY_IMPL(torchscience, AutocastCUDA, m) { m.impl(#name, tsbh::ops::name##_autocast); }

// --------------------------------------------------------------- binary ops
#define TSBH_BINARY_OP_CORE(name, Cls, A, B, FWD, BWD, BB)                                                   \
  namespace tsbh::ops {                                                                                 \
  at::Tensor name##_cuda(const at::Tensor& a, const at::Tensor& b) {                                   \
    return run_pointwise(FWD, #name, {a, b}, 1)[0];                                                    \
  }                                                                                                     \
  std::tuple<at::Tensor, at::Tensor> name##_backward_cuda(const at::Tensor& g, const at::Tensor& a,    \
                                                           const at::Tensor& b) {                      \
    auto r = run_pointwise(BWD, #name "_backward", {g, a, b}, 2);                                      \
    return {r[0], r[1]};                                                                               \
  }                                                                                                     \
  std::tuple<at::Tensor, at::Tensor, at::Tensor> name##_backward_backward_cuda(                        \
      const at::Tensor& gga, const at::Tensor& ggb, const at::Tensor& g, const at::Tensor& a, const at::Tensor& b) { \
    auto r = run_pointwise(BB, #name "_backward_backward", {gga, ggb, g, a, b}, 3);                   \
    return {r[0], r[1], r[2]};                                                                         \
  }                                                                                                     \
  at::Tensor name##_meta(const at::Tensor& a, const at::Tensor& b) {                                   \
    return meta_pointwise(#name, {a, b}, 1)[0];                                                        \
  }                                                                                                     \
  std::tuple<at::Tensor, at::Tensor> name##_backward_meta(const at::Tensor& g, const at::Tensor& a,    \
                                                           const at::Tensor& b) {                      \
    auto r = meta_pointwise(#name "_backward", {g, a, b}, 2);                                          \
    return {r[0], r[1]};                                                                               \
  }                                                                                                     \
  std::tuple<at::Tensor, at::Tensor, at::Tensor> name##_backward_backward_meta(                        \
      const at::Tensor& gga, const at::Tensor& ggb, const at::Tensor& g, const at::Tensor& a, const at::Tensor& b) { \
    auto r = meta_pointwise(#name "_backward_backward", {gga, ggb, g, a, b}, 3);                      \
    return {r[0], r[1], r[2]};                                                                         \
  }                                                                                                     \
  at::Tensor name##_cpu(const at::Tensor&, const at::Tensor&) { cpu_not_supported(#name); }            \
  std::tuple<at::Tensor, at::Tensor> name##_backward_cpu(const at::Tensor&, const at::Tensor&, const at::Tensor&) { \
    cpu_not_supported(#name "_backward");                                                              \
  }                                                                                                     \
  std::tuple<at::Tensor, at::Tensor, at::Tensor> name##_backward_backward_cpu(                         \
      const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&) { \
    cpu_not_supported(#name "_backward_backward");                                                     \
  }                                                                                                     \
  class Cls##Backward : public torch::autograd::Function<Cls##Backward> {                              \
   public:                                                                                              \
    static variable_list forward(AutogradContext* ctx, const at::Tensor& g, const at::Tensor& a,       \
                                 const at::Tensor& b, bool ra, bool rb) {                              \
      ctx->save_for_backward({g, a, b});                                                               \
      ctx->saved_data["ra"] = ra;                                                                      \
      ctx->saved_data["rb"] = rb;                                                                      \
      at::AutoDispatchBelowAutograd guard;                                                             \
      if (any_cuda({g, a, b}) && !any_traced({g, a, b})) {                                             \
        /* Gradients come back already reduced to a's and b's shapes. */                               \
        return defined_or_zero(run_reduced_backward(BWD, #name "_backward", g, {a, b}, {ra, rb}), {a, b}); \
      }                                                                                                 \
      static auto op = c10::Dispatcher::singleton()                                                    \
                           .findSchemaOrThrow("torchscience::" #name "_backward", "")                  \
                           .typed<std::tuple<at::Tensor, at::Tensor>(const at::Tensor&, const at::Tensor&, \
                                                                     const at::Tensor&)>();           \
      auto [ga, gb] = op.call(g, a, b);                                                                \
      return {ga, gb};                                                                                 \
    }                                                                                                   \
    static variable_list backward(AutogradContext* ctx, const variable_list& go) {                     \
      auto saved = ctx->get_saved_variables();                                                          \
      const bool ra = ctx->saved_data["ra"].toBool(), rb = ctx->saved_data["rb"].toBool();             \
      if ((!go[0].defined() && !go[1].defined()) || (!ra && !rb))                                      \
        return {at::Tensor(), at::Tensor(), at::Tensor(), at::Tensor(), at::Tensor()};                 \
      at::AutoDispatchBelowAutograd guard;                                                             \
      auto gga = go[0].defined() ? go[0] : at::zeros_like(saved[1]);                                   \
      auto ggb = go[1].defined() ? go[1] : at::zeros_like(saved[2]);                                   \
      static auto op = c10::Dispatcher::singleton()                                                    \
                           .findSchemaOrThrow("torchscience::" #name "_backward_backward", "")         \
                           .typed<std::tuple<at::Tensor, at::Tensor, at::Tensor>(                      \
                               const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&, \
                               const at::Tensor&)>();                                                  \
      auto [gg_out, g_a, g_b] = op.call(gga, ggb, saved[0], saved[1], saved[2]);                       \
      return {gg_out, g_a, g_b, at::Tensor(), at::Tensor()};                                           \
    }                                                                                                   \
  };                                                                                                    \
  class Cls : public torch::autograd::Function<Cls> {                                                  \
   public:                                                                                              \
    static at::Tensor forward(AutogradContext* ctx, const at::Tensor& a, const at::Tensor& b) {        \
      ctx->save_for_backward({a, b});                                                                  \
      ctx->saved_data["ra"] = wants_grad(a);                                                           \
      ctx->saved_data["rb"] = wants_grad(b);                                                           \
      at::AutoDispatchBelowAutograd guard;                                                             \
      static auto op = c10::Dispatcher::singleton()                                                    \
                           .findSchemaOrThrow("torchscience::" #name, "")                              \
                           .typed<at::Tensor(const at::Tensor&, const at::Tensor&)>();                 \
      return op.call(a, b);                                                                            \
    }                                                                                                   \
    static variable_list backward(AutogradContext* ctx, const variable_list& go) {                     \
      auto saved = ctx->get_saved_variables();                                                          \
      const bool ra = ctx->saved_data["ra"].toBool(), rb = ctx->saved_data["rb"].toBool();             \
      auto g = Cls##Backward::apply(go[0], saved[0], saved[1], ra, rb);                                \
      return {ra ? g[0] : at::Tensor(), rb ? g[1] : at::Tensor()};                                     \
    }                                                                                                   \
  };                                                                                                    \
  at::Tensor name##_autograd(const at::Tensor& a, const at::Tensor& b) { return Cls::apply(a, b); }     \
  at::Tensor name##_autocast(const at::Tensor& a, const at::Tensor& b) {                               \
    c10::impl::ExcludeDispatchKeyGuard no_autocast(c10::DispatchKey::AutocastCUDA);                    \
    const auto t = at::autocast::promote_type(at::kFloat, c10::DeviceType::CUDA, a, b);                \
    static auto op = c10::Dispatcher::singleton()                                                      \
                         .findSchemaOrThrow("torchscience::" #name, "")                                \
                         .typed<at::Tensor(const at::Tensor&, const at::Tensor&)>();                   \
    return op.call(at::autocast::cached_cast(t, a, c10::DeviceType::CUDA),                             \
                   at::autocast::cached_cast(t, b, c10::DeviceType::CUDA));                            \
  }                                                                                                     \
  } /* namespace tsbh::ops */                                                                           \
  TORCH_LIBRARY_IMPL(torchscience, CUDA, m) {                                                           \
    m.impl(#name, tsbh::ops::name##_cuda);                                                              \
    m.impl(#name "_backward", tsbh::ops::name##_backward_cuda);                                         \
    m.impl(#name "_backward_backward", tsbh::ops::name##_backward_backward_cuda);                       \
  }                                                                                                     \
  TORCH_LIBRARY_IMPL(torchscience, Meta, m) {                                                           \
    m.impl(#name, tsbh::ops::name##_meta);                                                              \
    m.impl(#name "_backward", tsbh::ops::name##_backward_meta);                                         \
    m.impl(#name "_backward_backward", tsbh::ops::name##_backward_backward_meta);                       \
  }                                                                                                     \
  TORCH_LIBRARY_IMPL(torchscience, CPU, m) {                                                            \
    m.impl(#name, tsbh::ops::name##_cpu);                                                               \
    m.impl(#name "_backward", tsbh::ops::name##_backward_cpu);                                          \
    m.impl(#name "_backward_backward", tsbh::ops::name##_backward_backward_cpu);                        \
  }                                                                                                     \
  TORCH_LIBRARY_IMPL(torchscience, AutocastCUDA, m) { m.impl(#name, tsbh::ops::name##_autocast); }
#define TSBH_BINARY_OP(name, Cls, A, B, FWD, BWD, BB)     \
  TSBH_BINARY_OP_CORE(name, Cls, A, B, FWD, BWD, BB)      \
  TORCH_LIBRARY_IMPL(torchscience, Autograd, m) { m.impl(#name, tsbh::ops::name##_autograd); }

// Autograd for P and Q: when an input requires grad on CUDA, the forward runs
// the fused kernel (value and first derivatives in one evaluation) and keeps
// the derivatives; the backward multiplies them by the incoming gradient and
// reduces to the inputs' shapes (an HBM-bound pass instead of a second
// evaluation).  Double backward is unchanged: the _backward_backward op from
// the saved inputs.  Without grad (no input requiring it, or grad mode off),
// or off CUDA, the plain forward runs.
#define TSBH_IGAMMA_FUSED_AUTOGRAD(name, Cls, FWDGRAD)                                                           \
  namespace tsbh::ops {                                                                                          \
  class Cls##SavedBackward : public torch::autograd::Function<Cls##SavedBackward> {                              \
   public:                                                                                                       \
    static variable_list forward(AutogradContext* ctx, const at::Tensor& g, const at::Tensor& a,                \
                                 const at::Tensor& b, const at::Tensor& da, const at::Tensor& db, bool ra,      \
                                 bool rb) {                                                                      \
      ctx->save_for_backward({g, a, b});                                                                        \
      ctx->saved_data["ra"] = ra;                                                                               \
      ctx->saved_data["rb"] = rb;                                                                               \
      at::AutoDispatchBelowAutograd guard;                                                                      \
      return defined_or_zero(run_reduced(tsb_gradient_product, #name "_backward", {g, da, db}, {a, b}, {ra, rb}), \
                             {a, b});                                                                           \
    }                                                                                                            \
    static variable_list backward(AutogradContext* ctx, const variable_list& go) {                              \
      auto saved = ctx->get_saved_variables();                                                                   \
      const bool ra = ctx->saved_data["ra"].toBool(), rb = ctx->saved_data["rb"].toBool();                      \
      const at::Tensor none;                                                                                     \
      if ((!go[0].defined() && !go[1].defined()) || (!ra && !rb)) return {none, none, none, none, none, none, none}; \
      at::AutoDispatchBelowAutograd guard;                                                                      \
      auto gga = go[0].defined() ? go[0] : at::zeros_like(saved[1]);                                            \
      auto ggb = go[1].defined() ? go[1] : at::zeros_like(saved[2]);                                            \
      static auto op = c10::Dispatcher::singleton()                                                             \
                           .findSchemaOrThrow("torchscience::" #name "_backward_backward", "")                  \
                           .typed<std::tuple<at::Tensor, at::Tensor, at::Tensor>(                               \
                               const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&,      \
                               const at::Tensor&)>();                                                           \
      auto [gg_out, g_a, g_b] = op.call(gga, ggb, saved[0], saved[1], saved[2]);                                \
      return {gg_out, g_a, g_b, none, none, none, none};                                                        \
    }                                                                                                            \
  };                                                                                                             \
  class Cls##Fused : public torch::autograd::Function<Cls##Fused> {                                              \
   public:                                                                                                       \
    static at::Tensor forward(AutogradContext* ctx, const at::Tensor& a, const at::Tensor& b, bool recorded) {  \
      const bool ra = wants_grad(a), rb = wants_grad(b);                                                        \
      ctx->saved_data["ra"] = ra;                                                                               \
      ctx->saved_data["rb"] = rb;                                                                               \
      at::AutoDispatchBelowAutograd guard;                                                                      \
      if ((ra || rb) && recorded && keep_derivatives().load() && any_cuda({a, b}) && !any_traced({a, b})) {    \
        auto r = run_pointwise_masked(FWDGRAD, #name, {a, b}, 3, {true, ra, rb});                               \
        ctx->save_for_backward({a, b, r[1], r[2]});                                                             \
        ctx->saved_data["fused"] = true;                                                                        \
        return r[0];                                                                                             \
      }                                                                                                          \
      ctx->save_for_backward({a, b});                                                                           \
      ctx->saved_data["fused"] = false;                                                                         \
      static auto op = c10::Dispatcher::singleton()                                                             \
                           .findSchemaOrThrow("torchscience::" #name, "")                                       \
                           .typed<at::Tensor(const at::Tensor&, const at::Tensor&)>();                          \
      return op.call(a, b);                                                                                      \
    }                                                                                                            \
    static variable_list backward(AutogradContext* ctx, const variable_list& go) {                              \
      auto saved = ctx->get_saved_variables();                                                                   \
      const bool ra = ctx->saved_data["ra"].toBool(), rb = ctx->saved_data["rb"].toBool();                      \
      if (!go[0].defined()) return {at::Tensor(), at::Tensor(), at::Tensor()};                                  \
      if (!ctx->saved_data["fused"].toBool()) {                                                                 \
        auto g = Cls##Backward::apply(go[0], saved[0], saved[1], ra, rb);                                        \
        return {ra ? g[0] : at::Tensor(), rb ? g[1] : at::Tensor(), at::Tensor()};                              \
      }                                                                                                          \
      /* an unwanted derivative was not kept: the other stands in (autograd Functions take no undefined      */ \
      /* tensors), and its product is skipped                                                                 */ \
      const at::Tensor& d0 = saved[2].defined() ? saved[2] : saved[3];                                           \
      const at::Tensor& d1 = saved[3].defined() ? saved[3] : saved[2];                                           \
      auto g = Cls##SavedBackward::apply(go[0], saved[0], saved[1], d0, d1, ra, rb);                             \
      return {ra ? g[0] : at::Tensor(), rb ? g[1] : at::Tensor(), at::Tensor()};                                \
    }                                                                                                            \
  };                                                                                                             \
  /* under no_grad the autograd kernel still runs, and apply() turns grad mode off before forward(): */           \
  /* whether this call is recorded is read here                                                       */           \
  at::Tensor name##_fused_autograd(const at::Tensor& a, const at::Tensor& b) {                                  \
    return Cls##Fused::apply(a, b, c10::GradMode::is_enabled());                                                \
  }                                                                                                              \
  } /* namespace tsbh::ops */                                                                                    \
  TORCH_LIBRARY_IMPL(torchscience, Autograd, m) { m.impl(#name, tsbh::ops::name##_fused_autograd); }

// Schemas: identical strings to the reference's TORCH_LIBRARY block.
TORCH_LIBRARY(torchscience, m) { TSB_DEFINE_TORCHSCIENCE_SCHEMAS(m) }

TSBH_UNARY_OP(log_gamma, LogGamma, z, tsb_log_gamma, tsb_log_gamma_backward, tsb_log_gamma_backward_backward)
TSBH_UNARY_OP(gamma, Gamma, z, tsb_gamma, tsb_gamma_backward, tsb_gamma_backward_backward)
TSBH_UNARY_OP(digamma, Digamma, z, tsb_digamma, tsb_digamma_backward, tsb_digamma_backward_backward)
TSBH_UNARY_OP(trigamma, Trigamma, z, tsb_trigamma, tsb_trigamma_backward, tsb_trigamma_backward_backward)
TSBH_BINARY_OP_CORE(regularized_gamma_p, RegularizedGammaP, a, x, tsb_regularized_gamma_p,
                    tsb_regularized_gamma_p_backward, tsb_regularized_gamma_p_backward_backward)
TSBH_IGAMMA_FUSED_AUTOGRAD(regularized_gamma_p, RegularizedGammaP, tsb_regularized_gamma_p_forward_with_grads)
TSBH_BINARY_OP_CORE(regularized_gamma_q, RegularizedGammaQ, a, x, tsb_regularized_gamma_q,
                    tsb_regularized_gamma_q_backward, tsb_regularized_gamma_q_backward_backward)
TSBH_IGAMMA_FUSED_AUTOGRAD(regularized_gamma_q, RegularizedGammaQ, tsb_regularized_gamma_q_forward_with_grads)
TSBH_BINARY_OP(polygamma, Polygamma, n, z, tsb_polygamma, tsb_polygamma_backward, tsb_polygamma_backward_backward)
TSBH_BINARY_OP(log_beta, LogBeta, a, b, tsb_log_beta, tsb_log_beta_backward, tsb_log_beta_backward_backward)
TSBH_BINARY_OP(beta, Beta, a, b, tsb_beta, tsb_beta_backward, tsb_beta_backward_backward)
TSBH_UNARY_OP(bessel_j_0, BesselJ0, z, tsb_bessel_j_0, tsb_bessel_j_0_backward, tsb_bessel_j_0_backward_backward)
TSBH_UNARY_OP(bessel_j_1, BesselJ1, z, tsb_bessel_j_1, tsb_bessel_j_1_backward, tsb_bessel_j_1_backward_backward)
TSBH_UNARY_OP(bessel_y_0, BesselY0, z, tsb_bessel_y_0, tsb_bessel_y_0_backward, tsb_bessel_y_0_backward_backward)
TSBH_UNARY_OP(bessel_y_1, BesselY1, z, tsb_bessel_y_1, tsb_bessel_y_1_backward, tsb_bessel_y_1_backward_backward)
TSBH_UNARY_OP(modified_bessel_i_0, ModifiedBesselI0, z, tsb_modified_bessel_i_0, tsb_modified_bessel_i_0_backward, tsb_modified_bessel_i_0_backward_backward)
TSBH_UNARY_OP(modified_bessel_i_1, ModifiedBesselI1, z, tsb_modified_bessel_i_1, tsb_modified_bessel_i_1_backward, tsb_modified_bessel_i_1_backward_backward)
TSBH_UNARY_OP(modified_bessel_k_0, ModifiedBesselK0, z, tsb_modified_bessel_k_0, tsb_modified_bessel_k_0_backward, tsb_modified_bessel_k_0_backward_backward)
TSBH_UNARY_OP(modified_bessel_k_1, ModifiedBesselK1, z, tsb_modified_bessel_k_1, tsb_modified_bessel_k_1_backward, tsb_modified_bessel_k_1_backward_backward)
TSBH_UNARY_OP(spherical_bessel_j_0, SphericalBesselJ0, z, tsb_spherical_bessel_j_0, tsb_spherical_bessel_j_0_backward, tsb_spherical_bessel_j_0_backward_backward)
TSBH_UNARY_OP(spherical_bessel_j_1, SphericalBesselJ1, z, tsb_spherical_bessel_j_1, tsb_spherical_bessel_j_1_backward, tsb_spherical_bessel_j_1_backward_backward)
TSBH_UNARY_OP(spherical_bessel_y_0, SphericalBesselY0, z, tsb_spherical_bessel_y_0, tsb_spherical_bessel_y_0_backward, tsb_spherical_bessel_y_0_backward_backward)
TSBH_UNARY_OP(spherical_bessel_y_1, SphericalBesselY1, z, tsb_spherical_bessel_y_1, tsb_spherical_bessel_y_1_backward, tsb_spherical_bessel_y_1_backward_backward)
TSBH_UNARY_OP(spherical_bessel_i_0, SphericalBesselI0, z, tsb_spherical_bessel_i_0, tsb_spherical_bessel_i_0_backward, tsb_spherical_bessel_i_0_backward_backward)
TSBH_UNARY_OP(spherical_bessel_i_1, SphericalBesselI1, z, tsb_spherical_bessel_i_1, tsb_spherical_bessel_i_1_backward, tsb_spherical_bessel_i_1_backward_backward)
TSBH_UNARY_OP(spherical_bessel_k_0, SphericalBesselK0, z, tsb_spherical_bessel_k_0, tsb_spherical_bessel_k_0_backward, tsb_spherical_bessel_k_0_backward_backward)
TSBH_UNARY_OP(spherical_bessel_k_1, SphericalBesselK1, z, tsb_spherical_bessel_k_1, tsb_spherical_bessel_k_1_backward, tsb_spherical_bessel_k_1_backward_backward)
TSBH_BINARY_OP(spherical_bessel_j, SphericalBesselJ, n, z, tsb_spherical_bessel_j, tsb_spherical_bessel_j_backward, tsb_spherical_bessel_j_backward_backward)
TSBH_BINARY_OP(spherical_bessel_y, SphericalBesselY, n, z, tsb_spherical_bessel_y, tsb_spherical_bessel_y_backward, tsb_spherical_bessel_y_backward_backward)
TSBH_BINARY_OP(spherical_bessel_i, SphericalBesselI, n, z, tsb_spherical_bessel_i, tsb_spherical_bessel_i_backward, tsb_spherical_bessel_i_backward_backward)
TSBH_BINARY_OP(spherical_bessel_k, SphericalBesselK, n, z, tsb_spherical_bessel_k, tsb_spherical_bessel_k_backward, tsb_spherical_bessel_k_backward_backward)
TSBH_BINARY_OP(bessel_j, BesselJ, n, z, tsb_bessel_j, tsb_bessel_j_backward, tsb_bessel_j_backward_backward)
TSBH_BINARY_OP(bessel_y, BesselY, n, z, tsb_bessel_y, tsb_bessel_y_backward, tsb_bessel_y_backward_backward)
TSBH_BINARY_OP(modified_bessel_i, ModifiedBesselI, n, z, tsb_modified_bessel_i, tsb_modified_bessel_i_backward,
               tsb_modified_bessel_i_backward_backward)
TSBH_BINARY_OP(modified_bessel_k, ModifiedBesselK, n, z, tsb_modified_bessel_k, tsb_modified_bessel_k_backward,
               tsb_modified_bessel_k_backward_backward)
TSBH_UNARY_OP(complete_legendre_elliptic_integral_k, CompleteLegendreEllipticIntegralK, m,
              tsb_complete_legendre_elliptic_integral_k, tsb_complete_legendre_elliptic_integral_k_backward,
              tsb_complete_legendre_elliptic_integral_k_backward_backward)
TSBH_UNARY_OP(complete_legendre_elliptic_integral_e, CompleteLegendreEllipticIntegralE, m,
              tsb_complete_legendre_elliptic_integral_e, tsb_complete_legendre_elliptic_integral_e_backward,
              tsb_complete_legendre_elliptic_integral_e_backward_backward)

// ------------------------------------------------------------ 2F1(a, b; c; z)
// The one quaternary op (reference CPU loop: cpu/macros.h:2905; autograd
// structure as the binary ops above, with four inputs).
namespace tsbh::ops {
using T4 = std::tuple<at::Tensor, at::Tensor, at::Tensor, at::Tensor>;
using T5 = std::tuple<at::Tensor, at::Tensor, at::Tensor, at::Tensor, at::Tensor>;

at::Tensor hyp2f1_cuda(const at::Tensor& a, const at::Tensor& b, const at::Tensor& c, const at::Tensor& z) {
  return run_pointwise(tsb_hypergeometric_2_f_1, "hypergeometric_2_f_1", {a, b, c, z}, 1)[0];
}
T4 hyp2f1_backward_cuda(const at::Tensor& g, const at::Tensor& a, const at::Tensor& b, const at::Tensor& c,
                        const at::Tensor& z) {
  auto r = run_pointwise(tsb_hypergeometric_2_f_1_backward, "hypergeometric_2_f_1_backward", {g, a, b, c, z}, 4);
  return {r[0], r[1], r[2], r[3]};
}
T5 hyp2f1_backward_backward_cuda(const at::Tensor& gga, const at::Tensor& ggb, const at::Tensor& ggc,
                                 const at::Tensor& ggz, const at::Tensor& g, const at::Tensor& a, const at::Tensor& b,
                                 const at::Tensor& c, const at::Tensor& z) {
  auto r = run_pointwise(tsb_hypergeometric_2_f_1_backward_backward, "hypergeometric_2_f_1_backward_backward",
                         {gga, ggb, ggc, ggz, g, a, b, c, z}, 5);
  return {r[0], r[1], r[2], r[3], r[4]};
}
at::Tensor hyp2f1_meta(const at::Tensor& a, const at::Tensor& b, const at::Tensor& c, const at::Tensor& z) {
  return meta_pointwise("hypergeometric_2_f_1", {a, b, c, z}, 1)[0];
}
T4 hyp2f1_backward_meta(const at::Tensor& g, const at::Tensor& a, const at::Tensor& b, const at::Tensor& c,
                        const at::Tensor& z) {
  auto r = meta_pointwise("hypergeometric_2_f_1_backward", {g, a, b, c, z}, 4);
  return {r[0], r[1], r[2], r[3]};
}
T5 hyp2f1_backward_backward_meta(const at::Tensor& gga, const at::Tensor& ggb, const at::Tensor& ggc,
                                 const at::Tensor& ggz, const at::Tensor& g, const at::Tensor& a, const at::Tensor& b,
                                 const at::Tensor& c, const at::Tensor& z) {
  auto r = meta_pointwise("hypergeometric_2_f_1_backward_backward", {gga, ggb, ggc, ggz, g, a, b, c, z}, 5);
  return {r[0], r[1], r[2], r[3], r[4]};
}
at::Tensor hyp2f1_cpu(const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&) {
  cpu_not_supported("hypergeometric_2_f_1");
}
T4 hyp2f1_backward_cpu(const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&,
                       const at::Tensor&) {
  cpu_not_supported("hypergeometric_2_f_1_backward");
}
T5 hyp2f1_backward_backward_cpu(const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&,
                                const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&,
                                const at::Tensor&) {
  cpu_not_supported("hypergeometric_2_f_1_backward_backward");
}

class Hypergeometric2F1Backward : public torch::autograd::Function<Hypergeometric2F1Backward> {
 public:
  static variable_list forward(AutogradContext* ctx, const at::Tensor& g, const at::Tensor& a, const at::Tensor& b,
                               const at::Tensor& c, const at::Tensor& z, std::vector<bool> want) {
    ctx->save_for_backward({g, a, b, c, z});
    for (int i = 0; i < 4; ++i) ctx->saved_data["r" + std::to_string(i)] = static_cast<bool>(want[i]);
    at::AutoDispatchBelowAutograd guard;
    if (any_cuda({g, a, b, c, z}) && !any_traced({g, a, b, c, z})) {
      /* Gradients come back already reduced to the inputs' shapes. */
      return defined_or_zero(run_reduced_backward(tsb_hypergeometric_2_f_1_backward, "hypergeometric_2_f_1_backward",
                                                  g, {a, b, c, z}, want),
                             {a, b, c, z});
    }
    static auto op = c10::Dispatcher::singleton()
                         .findSchemaOrThrow("torchscience::hypergeometric_2_f_1_backward", "")
                         .typed<T4(const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&,
                                   const at::Tensor&)>();
    auto [ga, gb, gc, gz] = op.call(g, a, b, c, z);
    return {ga, gb, gc, gz};
  }
  static variable_list backward(AutogradContext* ctx, const variable_list& go) {
    auto saved = ctx->get_saved_variables();
    bool any_req = false, any_go = false;
    for (int i = 0; i < 4; ++i) {
      any_req = any_req || ctx->saved_data["r" + std::to_string(i)].toBool();
      any_go = any_go || go[i].defined();
    }
    variable_list none(7);
    if (!any_go || !any_req) return none;
    at::AutoDispatchBelowAutograd guard;
    at::Tensor gg[4];
    for (int i = 0; i < 4; ++i) gg[i] = go[i].defined() ? go[i] : at::zeros_like(saved[1 + i]);
    static auto op = c10::Dispatcher::singleton()
                         .findSchemaOrThrow("torchscience::hypergeometric_2_f_1_backward_backward", "")
                         .typed<T5(const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&,
                                   const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&,
                                   const at::Tensor&)>();
    auto [gg_out, g_a, g_b, g_c, g_z] =
        op.call(gg[0], gg[1], gg[2], gg[3], saved[0], saved[1], saved[2], saved[3], saved[4]);
    return {gg_out, g_a, g_b, g_c, g_z, at::Tensor()};
  }
};

class Hypergeometric2F1 : public torch::autograd::Function<Hypergeometric2F1> {
 public:
  static at::Tensor forward(AutogradContext* ctx, const at::Tensor& a, const at::Tensor& b, const at::Tensor& c,
                            const at::Tensor& z) {
    ctx->save_for_backward({a, b, c, z});
    const at::Tensor* in[4] = {&a, &b, &c, &z};
    for (int i = 0; i < 4; ++i) ctx->saved_data["r" + std::to_string(i)] = wants_grad(*in[i]);
    at::AutoDispatchBelowAutograd guard;
    static auto op = c10::Dispatcher::singleton()
                         .findSchemaOrThrow("torchscience::hypergeometric_2_f_1", "")
                         .typed<at::Tensor(const at::Tensor&, const at::Tensor&, const at::Tensor&,
                                           const at::Tensor&)>();
    return op.call(a, b, c, z);
  }
  static variable_list backward(AutogradContext* ctx, const variable_list& go) {
    auto saved = ctx->get_saved_variables();
    std::vector<bool> want(4);
    for (int i = 0; i < 4; ++i) want[i] = ctx->saved_data["r" + std::to_string(i)].toBool();
    auto g = Hypergeometric2F1Backward::apply(go[0], saved[0], saved[1], saved[2], saved[3], want);
    variable_list out(4);
    for (int i = 0; i < 4; ++i) out[i] = want[i] ? g[i] : at::Tensor();
    return out;
  }
};

at::Tensor hyp2f1_autograd(const at::Tensor& a, const at::Tensor& b, const at::Tensor& c, const at::Tensor& z) {
  return Hypergeometric2F1::apply(a, b, c, z);
}
at::Tensor hyp2f1_autocast(const at::Tensor& a, const at::Tensor& b, const at::Tensor& c, const at::Tensor& z) {
  c10::impl::ExcludeDispatchKeyGuard no_autocast(c10::DispatchKey::AutocastCUDA);
  const auto t = at::autocast::promote_type(at::kFloat, c10::DeviceType::CUDA, a, b, c, z);
  static auto op = c10::Dispatcher::singleton()
                       .findSchemaOrThrow("torchscience::hypergeometric_2_f_1", "")
                       .typed<at::Tensor(const at::Tensor&, const at::Tensor&, const at::Tensor&,
                                         const at::Tensor&)>();
  const auto dev = c10::DeviceType::CUDA;
  return op.call(at::autocast::cached_cast(t, a, dev), at::autocast::cached_cast(t, b, dev),
                 at::autocast::cached_cast(t, c, dev), at::autocast::cached_cast(t, z, dev));
}
}  // namespace tsbh::ops

TORCH_LIBRARY_IMPL(torchscience, CUDA, m) {
  m.impl("hypergeometric_2_f_1", tsbh::ops::hyp2f1_cuda);
  m.impl("hypergeometric_2_f_1_backward", tsbh::ops::hyp2f1_backward_cuda);
  m.impl("hypergeometric_2_f_1_backward_backward", tsbh::ops::hyp2f1_backward_backward_cuda);
}
TORCH_LIBRARY_IMPL(torchscience, Meta, m) {
  m.impl("hypergeometric_2_f_1", tsbh::ops::hyp2f1_meta);
  m.impl("hypergeometric_2_f_1_backward", tsbh::ops::hyp2f1_backward_meta);
  m.impl("hypergeometric_2_f_1_backward_backward", tsbh::ops::hyp2f1_backward_backward_meta);
}
TORCH_LIBRARY_IMPL(torchscience, CPU, m) {
  m.impl("hypergeometric_2_f_1", tsbh::ops::hyp2f1_cpu);
  m.impl("hypergeometric_2_f_1_backward", tsbh::ops::hyp2f1_backward_cpu);
  m.impl("hypergeometric_2_f_1_backward_backward", tsbh::ops::hyp2f1_backward_backward_cpu);
}
TORCH_LIBRARY_IMPL(torchscience, Autograd, m) { m.impl("hypergeometric_2_f_1", tsbh::ops::hyp2f1_autograd); }
TORCH_LIBRARY_IMPL(torchscience, AutocastCUDA, m) { m.impl("hypergeometric_2_f_1", tsbh::ops::hyp2f1_autocast); }

// ------------------------------------------------------------- I_x(a, b)
// The one ternary special function (autograd structure as the binary ops
// above, with three inputs).
namespace tsbh::ops {
using T3i = std::tuple<at::Tensor, at::Tensor, at::Tensor>;
using T4i = std::tuple<at::Tensor, at::Tensor, at::Tensor, at::Tensor>;

at::Tensor ibeta_cuda(const at::Tensor& x, const at::Tensor& a, const at::Tensor& b) {
  return run_pointwise(tsb_incomplete_beta, "incomplete_beta", {x, a, b}, 1)[0];
}
T3i ibeta_backward_cuda(const at::Tensor& g, const at::Tensor& x, const at::Tensor& a, const at::Tensor& b) {
  auto r = run_pointwise(tsb_incomplete_beta_backward, "incomplete_beta_backward", {g, x, a, b}, 3);
  return {r[0], r[1], r[2]};
}
T4i ibeta_backward_backward_cuda(const at::Tensor& ggx, const at::Tensor& gga, const at::Tensor& ggb,
                                 const at::Tensor& g, const at::Tensor& x, const at::Tensor& a, const at::Tensor& b) {
  auto r = run_pointwise(tsb_incomplete_beta_backward_backward, "incomplete_beta_backward_backward",
                         {ggx, gga, ggb, g, x, a, b}, 4);
  return {r[0], r[1], r[2], r[3]};
}
at::Tensor ibeta_meta(const at::Tensor& x, const at::Tensor& a, const at::Tensor& b) {
  return meta_pointwise("incomplete_beta", {x, a, b}, 1)[0];
}
T3i ibeta_backward_meta(const at::Tensor& g, const at::Tensor& x, const at::Tensor& a, const at::Tensor& b) {
  auto r = meta_pointwise("incomplete_beta_backward", {g, x, a, b}, 3);
  return {r[0], r[1], r[2]};
}
T4i ibeta_backward_backward_meta(const at::Tensor& ggx, const at::Tensor& gga, const at::Tensor& ggb,
                                 const at::Tensor& g, const at::Tensor& x, const at::Tensor& a, const at::Tensor& b) {
  auto r = meta_pointwise("incomplete_beta_backward_backward", {ggx, gga, ggb, g, x, a, b}, 4);
  return {r[0], r[1], r[2], r[3]};
}
at::Tensor ibeta_cpu(const at::Tensor&, const at::Tensor&, const at::Tensor&) {
  cpu_not_supported("incomplete_beta");
}
T3i ibeta_backward_cpu(const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&) {
  cpu_not_supported("incomplete_beta_backward");
}
T4i ibeta_backward_backward_cpu(const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&,
                                const at::Tensor&, const at::Tensor&, const at::Tensor&) {
  cpu_not_supported("incomplete_beta_backward_backward");
}

class IncompleteBetaBackward : public torch::autograd::Function<IncompleteBetaBackward> {
 public:
  static variable_list forward(AutogradContext* ctx, const at::Tensor& g, const at::Tensor& x, const at::Tensor& a,
                               const at::Tensor& b, std::vector<bool> want) {
    ctx->save_for_backward({g, x, a, b});
    for (int i = 0; i < 3; ++i) ctx->saved_data["r" + std::to_string(i)] = static_cast<bool>(want[i]);
    at::AutoDispatchBelowAutograd guard;
    if (any_cuda({g, x, a, b}) && !any_traced({g, x, a, b})) {
      /* Gradients come back already reduced to the inputs' shapes; an
         unwanted output skips its work (only ∂x skips the fraction). */
      return defined_or_zero(
          run_reduced_backward(tsb_incomplete_beta_backward, "incomplete_beta_backward", g, {x, a, b}, want),
          {x, a, b});
    }
    static auto op = c10::Dispatcher::singleton()
                         .findSchemaOrThrow("torchscience::incomplete_beta_backward", "")
                         .typed<T3i(const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&)>();
    auto [gx, ga, gb] = op.call(g, x, a, b);
    return {gx, ga, gb};
  }
  static variable_list backward(AutogradContext* ctx, const variable_list& go) {
    auto saved = ctx->get_saved_variables();
    bool any_req = false, any_go = false;
    for (int i = 0; i < 3; ++i) {
      any_req = any_req || ctx->saved_data["r" + std::to_string(i)].toBool();
      any_go = any_go || go[i].defined();
    }
    variable_list none(5);
    if (!any_go || !any_req) return none;
    at::AutoDispatchBelowAutograd guard;
    at::Tensor gg[3];
    for (int i = 0; i < 3; ++i) gg[i] = go[i].defined() ? go[i] : at::zeros_like(saved[1 + i]);
    static auto op = c10::Dispatcher::singleton()
                         .findSchemaOrThrow("torchscience::incomplete_beta_backward_backward", "")
                         .typed<T4i(const at::Tensor&, const at::Tensor&, const at::Tensor&, const at::Tensor&,
                                    const at::Tensor&, const at::Tensor&, const at::Tensor&)>();
    auto [gg_out, g_x, g_a, g_b] = op.call(gg[0], gg[1], gg[2], saved[0], saved[1], saved[2], saved[3]);
    return {gg_out, g_x, g_a, g_b, at::Tensor()};
  }
};

class IncompleteBeta : public torch::autograd::Function<IncompleteBeta> {
 public:
  static at::Tensor forward(AutogradContext* ctx, const at::Tensor& x, const at::Tensor& a, const at::Tensor& b) {
    ctx->save_for_backward({x, a, b});
    const at::Tensor* in[3] = {&x, &a, &b};
    for (int i = 0; i < 3; ++i) ctx->saved_data["r" + std::to_string(i)] = wants_grad(*in[i]);
    at::AutoDispatchBelowAutograd guard;
    static auto op = c10::Dispatcher::singleton()
                         .findSchemaOrThrow("torchscience::incomplete_beta", "")
                         .typed<at::Tensor(const at::Tensor&, const at::Tensor&, const at::Tensor&)>();
    return op.call(x, a, b);
  }
  static variable_list backward(AutogradContext* ctx, const variable_list& go) {
    auto saved = ctx->get_saved_variables();
    std::vector<bool> want(3);
    for (int i = 0; i < 3; ++i) want[i] = ctx->saved_data["r" + std::to_string(i)].toBool();
    auto g = IncompleteBetaBackward::apply(go[0], saved[0], saved[1], saved[2], want);
    variable_list out(3);
    for (int i = 0; i < 3; ++i) out[i] = want[i] ? g[i] : at::Tensor();
    return out;
  }
};

at::Tensor ibeta_autograd(const at::Tensor& x, const at::Tensor& a, const at::Tensor& b) {
  return IncompleteBeta::apply(x, a, b);
}
at::Tensor ibeta_autocast(const at::Tensor& x, const at::Tensor& a, const at::Tensor& b) {
  c10::impl::ExcludeDispatchKeyGuard no_autocast(c10::DispatchKey::AutocastCUDA);
  const auto t = at::autocast::promote_type(at::kFloat, c10::DeviceType::CUDA, x, a, b);
  static auto op = c10::Dispatcher::singleton()
                       .findSchemaOrThrow("torchscience::incomplete_beta", "")
                       .typed<at::Tensor(const at::Tensor&, const at::Tensor&, const at::Tensor&)>();
  const auto dev = c10::DeviceType::CUDA;
  return op.call(at::autocast::cached_cast(t, x, dev), at::autocast::cached_cast(t, a, dev),
                 at::autocast::cached_cast(t, b, dev));
}
}  // namespace tsbh::ops

TORCH_LIBRARY_IMPL(torchscience, CUDA, m) {
  m.impl("incomplete_beta", tsbh::ops::ibeta_cuda);
  m.impl("incomplete_beta_backward", tsbh::ops::ibeta_backward_cuda);
  m.impl("incomplete_beta_backward_backward", tsbh::ops::ibeta_backward_backward_cuda);
}
TORCH_LIBRARY_IMPL(torchscience, Meta, m) {
  m.impl("incomplete_beta", tsbh::ops::ibeta_meta);
  m.impl("incomplete_beta_backward", tsbh::ops::ibeta_backward_meta);
  m.impl("incomplete_beta_backward_backward", tsbh::ops::ibeta_backward_backward_meta);
}
TORCH_LIBRARY_IMPL(torchscience, CPU, m) {
  m.impl("incomplete_beta", tsbh::ops::ibeta_cpu);
  m.impl("incomplete_beta_backward", tsbh::ops::ibeta_backward_cpu);
  m.impl("incomplete_beta_backward_backward", tsbh::ops::ibeta_backward_backward_cpu);
}
TORCH_LIBRARY_IMPL(torchscience, Autograd, m) { m.impl("incomplete_beta", tsbh::ops::ibeta_autograd); }
TORCH_LIBRARY_IMPL(torchscience, AutocastCUDA, m) { m.impl("incomplete_beta", tsbh::ops::ibeta_autocast); }

// ------------------------------------------- probability callers of P and Q
// gamma / chi2 / poisson cumulative distributions, the chi2 survival function
// and the gamma / chi2 densities (torchscience.cpp:1881-1924).  As in the
// reference (autograd/probability/*.h, cpu/probability/*.h), the backward ops
// return gradients already reduced to the inputs' shapes and have no double
// backward.  Each op gets CUDA, Meta, CPU (an error) and Autograd kernels from
// one macro per arity.
namespace tsbh::prob {
using T2 = std::tuple<at::Tensor, at::Tensor>;
using T3 = std::tuple<at::Tensor, at::Tensor, at::Tensor>;

inline std::vector<at::Tensor> meta_grads(at::TensorList ins) {
  at::ScalarType dt = ins[0].scalar_type();
  for (const auto& t : ins) dt = at::promote_types(dt, t.scalar_type());
  std::vector<at::Tensor> r;
  for (const auto& t : ins) r.push_back(at::empty(t.sizes(), t.options().dtype(dt).device(at::kMeta)));
  return r;
}
inline std::vector<at::Tensor> reduced_all(OpFn fn, const char* name, const at::Tensor& g, at::TensorList ins) {
  return run_reduced_backward(fn, name, g, ins, std::vector<bool>(ins.size(), true));
}
template <typename Sig>
inline auto op(const char* name) {
  return c10::Dispatcher::singleton().findSchemaOrThrow(name, "").typed<Sig>();
}
using A = const at::Tensor&;

#define TSB_PROB_OP2(ID, NAME)                                                                               \
  at::Tensor ID##_cuda(A a, A b) { return run_pointwise(tsb_##NAME, #NAME, {a, b}, 1)[0]; }                 \
  T2 ID##_backward_cuda(A g, A a, A b) {                                                                     \
    auto r = reduced_all(tsb_##NAME##_backward, #NAME "_backward", g, {a, b});                               \
    return {r[0], r[1]};                                                                                     \
  }                                                                                                          \
  at::Tensor ID##_meta(A a, A b) { return meta_pointwise(#NAME, {a, b}, 1)[0]; }                            \
  T2 ID##_backward_meta(A, A a, A b) {                                                                       \
    auto r = meta_grads({a, b});                                                                             \
    return {r[0], r[1]};                                                                                     \
  }                                                                                                          \
  at::Tensor ID##_cpu(A, A) { cpu_not_supported(#NAME); }                                                    \
  T2 ID##_backward_cpu(A, A, A) { cpu_not_supported(#NAME "_backward"); }                                    \
  class ID##_fn : public torch::autograd::Function<ID##_fn> {                                                \
   public:                                                                                                   \
    static at::Tensor forward(AutogradContext* ctx, A a, A b) {                                              \
      ctx->save_for_backward({a, b});                                                                        \
      at::AutoDispatchBelowAutograd guard;                                                                   \
      static auto f = op<at::Tensor(A, A)>("torchscience::" #NAME);                                          \
      return f.call(a, b);                                                                                   \
    }                                                                                                        \
    static variable_list backward(AutogradContext* ctx, const variable_list& go) {                           \
      auto s = ctx->get_saved_variables();                                                                   \
      if (!go[0].defined()) return {at::Tensor(), at::Tensor()};                                             \
      at::AutoDispatchBelowAutograd guard;                                                                   \
      static auto bw = op<T2(A, A, A)>("torchscience::" #NAME "_backward");                                  \
      auto [ga, gb] = bw.call(go[0], s[0], s[1]);                                                            \
      return {ga, gb};                                                                                       \
    }                                                                                                        \
  };                                                                                                         \
  at::Tensor ID##_autograd(A a, A b) { return ID##_fn::apply(a, b); }

#define TSB_PROB_OP3(ID, NAME)                                                                               \
  at::Tensor ID##_cuda(A a, A b, A c) { return run_pointwise(tsb_##NAME, #NAME, {a, b, c}, 1)[0]; }         \
  T3 ID##_backward_cuda(A g, A a, A b, A c) {                                                                \
    auto r = reduced_all(tsb_##NAME##_backward, #NAME "_backward", g, {a, b, c});                            \
    return {r[0], r[1], r[2]};                                                                               \
  }                                                                                                          \
  at::Tensor ID##_meta(A a, A b, A c) { return meta_pointwise(#NAME, {a, b, c}, 1)[0]; }                    \
  T3 ID##_backward_meta(A, A a, A b, A c) {                                                                  \
    auto r = meta_grads({a, b, c});                                                                          \
    return {r[0], r[1], r[2]};                                                                               \
  }                                                                                                          \
  at::Tensor ID##_cpu(A, A, A) { cpu_not_supported(#NAME); }                                                 \
  T3 ID##_backward_cpu(A, A, A, A) { cpu_not_supported(#NAME "_backward"); }                                 \
  class ID##_fn : public torch::autograd::Function<ID##_fn> {                                                \
   public:                                                                                                   \
    static at::Tensor forward(AutogradContext* ctx, A a, A b, A c) {                                         \
      ctx->save_for_backward({a, b, c});                                                                     \
      at::AutoDispatchBelowAutograd guard;                                                                   \
      static auto f = op<at::Tensor(A, A, A)>("torchscience::" #NAME);                                       \
      return f.call(a, b, c);                                                                                \
    }                                                                                                        \
    static variable_list backward(AutogradContext* ctx, const variable_list& go) {                           \
      auto s = ctx->get_saved_variables();                                                                   \
      if (!go[0].defined()) return {at::Tensor(), at::Tensor(), at::Tensor()};                               \
      at::AutoDispatchBelowAutograd guard;                                                                   \
      static auto bw = op<T3(A, A, A, A)>("torchscience::" #NAME "_backward");                               \
      auto [ga, gb, gc] = bw.call(go[0], s[0], s[1], s[2]);                                                  \
      return {ga, gb, gc};                                                                                   \
    }                                                                                                        \
  };                                                                                                         \
  at::Tensor ID##_autograd(A a, A b, A c) { return ID##_fn::apply(a, b, c); }

TSB_PROB_OP2(chi2_cdf, chi2_cumulative_distribution)
TSB_PROB_OP3(gamma_cdf, gamma_cumulative_distribution)
TSB_PROB_OP2(poisson_cdf, poisson_cumulative_distribution)
TSB_PROB_OP2(chi2_sf, chi2_survival)
TSB_PROB_OP3(gamma_pdf, gamma_probability_density)
TSB_PROB_OP2(chi2_pdf, chi2_probability_density)
#undef TSB_PROB_OP2
#undef TSB_PROB_OP3
}  // namespace tsbh::prob

#define TSB_PROB_IMPL(ID, NAME, KEY)                   \
  m.impl(#NAME, tsbh::prob::ID##_##KEY);              \
  m.impl(#NAME "_backward", tsbh::prob::ID##_backward_##KEY);
#define TSB_PROB_ALL(KEY)                                          \
  TSB_PROB_IMPL(chi2_cdf, chi2_cumulative_distribution, KEY)       \
  TSB_PROB_IMPL(gamma_cdf, gamma_cumulative_distribution, KEY)     \
  TSB_PROB_IMPL(poisson_cdf, poisson_cumulative_distribution, KEY) \
  TSB_PROB_IMPL(chi2_sf, chi2_survival, KEY)                       \
  TSB_PROB_IMPL(gamma_pdf, gamma_probability_density, KEY)         \
  TSB_PROB_IMPL(chi2_pdf, chi2_probability_density, KEY)

TORCH_LIBRARY_FRAGMENT(torchscience, m) { TSB_DEFINE_PROBABILITY_SCHEMAS(m) }
TORCH_LIBRARY_IMPL(torchscience, CUDA, m) { TSB_PROB_ALL(cuda) }
TORCH_LIBRARY_IMPL(torchscience, Meta, m) { TSB_PROB_ALL(meta) }
TORCH_LIBRARY_IMPL(torchscience, CPU, m) { TSB_PROB_ALL(cpu) }
TORCH_LIBRARY_IMPL(torchscience, Autograd, m) {
  m.impl("chi2_cumulative_distribution", tsbh::prob::chi2_cdf_autograd);
  m.impl("gamma_cumulative_distribution", tsbh::prob::gamma_cdf_autograd);
  m.impl("poisson_cumulative_distribution", tsbh::prob::poisson_cdf_autograd);
  m.impl("chi2_survival", tsbh::prob::chi2_sf_autograd);
  m.impl("gamma_probability_density", tsbh::prob::gamma_pdf_autograd);
  m.impl("chi2_probability_density", tsbh::prob::chi2_pdf_autograd);
}
#undef TSB_PROB_ALL
#undef TSB_PROB_IMPL

// Library-level controls (not part of the reference's namespace).
namespace tsbh {
int64_t set_precision_mode(int64_t mode) {
  TORCH_CHECK(mode == TSB_PRECISION_AUTO || mode == TSB_PRECISION_FP64, "precision mode must be 0 (auto) or 1 (fp64)");
  return precision_mode().exchange(static_cast<int>(mode));
}
int64_t get_precision_mode() { return precision_mode().load(); }
bool set_keep_derivatives(bool keep) { return keep_derivatives().exchange(keep); }
bool get_keep_derivatives() { return keep_derivatives().load(); }
std::string library_version() { return tsb_version(); }
}  // namespace tsbh

TORCH_LIBRARY(torchscience_b200, m) {
  m.def("set_precision_mode(int mode) -> int", &tsbh::set_precision_mode);
  m.def("get_precision_mode() -> int", &tsbh::get_precision_mode);
  m.def("set_keep_derivatives(bool keep) -> bool", &tsbh::set_keep_derivatives);
  m.def("get_keep_derivatives() -> bool", &tsbh::get_keep_derivatives);
  m.def("version() -> str", &tsbh::library_version);
}
