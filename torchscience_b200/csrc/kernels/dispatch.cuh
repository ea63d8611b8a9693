// Host-side dispatch shared by every C-ABI entry point: operand validation,
// dimension coalescing, reduced-output detection, precision/dtype selection,
// launch configuration and error reporting.
#pragma once

#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include <algorithm>

#include "map.cuh"
#include "sweep_decl.cuh"

namespace tsb {

// Sets the calling thread's error message; returns `status`.
int32_t set_error(int32_t status, const char* fmt, ...);
// Adds n to the process-wide count of launched kernels (tsb_launch_count).
void count_launches(int64_t n);

struct DeviceInfo {
  int sm_count;
  int major, minor;
  bool ok;
};
// Cached per device; checks for compute capability 10.0 (the sm_100a code in
// this library runs nowhere else).
int32_t current_device(int* dev, const DeviceInfo** info);

constexpr int kMaxOperands = 16;

// Coalesced iteration space over all operands (inputs first, then outputs).
struct Canon {
  int ndim;
  int64_t numel;
  int64_t size[kMaxDims];
  int64_t stride[kMaxOperands][kMaxDims];
};

inline int32_t dtype_size(int32_t dt) {
  switch (dt) {
    case TSB_F32: return 4;
    case TSB_F64: return 8;
    case TSB_F16: return 2;
    case TSB_BF16: return 2;
    case TSB_C64: return 8;
    case TSB_C128: return 16;
    default: return 0;
  }
}

// Validates operands and coalesces dims.  Outputs with data == NULL are
// skipped (their strides are ignored when merging).
inline int32_t canonicalize(const tsb_tensor* in, int32_t n_in, const tsb_tensor* out, int32_t n_out, int32_t nin_expect,
                            int32_t nout_expect, Canon& c, int32_t& dtype) {
  if (n_in != nin_expect || n_out != nout_expect)
    return set_error(TSB_ERR_ARGUMENT, "expected %d inputs and %d outputs, got %d and %d", nin_expect, nout_expect, n_in,
                     n_out);
  if (!in || !out) return set_error(TSB_ERR_ARGUMENT, "null operand array");
  const int nops = n_in + n_out;
  if (nops > kMaxOperands) return set_error(TSB_ERR_ARGUMENT, "too many operands");
  const tsb_tensor* ops[kMaxOperands];
  for (int i = 0; i < n_in; ++i) ops[i] = &in[i];
  for (int i = 0; i < n_out; ++i) ops[n_in + i] = &out[i];
  const int nd = in[0].ndim;
  if (nd < 0 || nd > kMaxDims) return set_error(TSB_ERR_ARGUMENT, "ndim %d out of range [0, %d]", nd, kMaxDims);
  dtype = in[0].dtype;
  if (dtype_size(dtype) == 0) return set_error(TSB_ERR_DTYPE, "unknown dtype code %d", dtype);
  for (int k = 0; k < nops; ++k) {
    const tsb_tensor& t = *ops[k];
    const bool is_out = k >= n_in;
    if (!is_out && !t.data) return set_error(TSB_ERR_ARGUMENT, "input %d has a null data pointer", k);
    if (!t.data) continue;
    if (t.dtype != dtype) return set_error(TSB_ERR_DTYPE, "operand %d has dtype %d, expected %d", k, t.dtype, dtype);
    if (t.ndim != nd) return set_error(TSB_ERR_ARGUMENT, "operand %d has ndim %d, expected %d", k, t.ndim, nd);
    for (int d = 0; d < nd; ++d) {
      if (t.sizes[d] != in[0].sizes[d])
        return set_error(TSB_ERR_ARGUMENT, "operand %d size[%d] = %lld differs from the iteration shape", k, d,
                         (long long)t.sizes[d]);
      if (is_out && t.strides[d] < 0)
        return set_error(TSB_ERR_ARGUMENT, "output %d has a negative stride", k - n_in);
    }
    const uintptr_t align = (uintptr_t)dtype_size(dtype);
    if (((uintptr_t)t.data) % align != 0) return set_error(TSB_ERR_ARGUMENT, "operand %d is misaligned", k);
  }
  // Drop size-1 dims, detect empty.
  c.numel = 1;
  c.ndim = 0;
  for (int d = 0; d < nd; ++d) {
    const int64_t s = in[0].sizes[d];
    if (s < 0) return set_error(TSB_ERR_ARGUMENT, "negative size");
    c.numel *= s;
    if (s == 1) continue;
    c.size[c.ndim] = s;
    for (int k = 0; k < nops; ++k) c.stride[k][c.ndim] = ops[k]->data ? ops[k]->strides[d] : 0;
    ++c.ndim;
  }
  if (c.numel == 0) return TSB_OK;
  // Merge adjacent dims (outer d, inner d+1) where every operand allows it.
  int w = 0;
  for (int d = 1; d < c.ndim; ++d) {
    bool ok = true;
    for (int k = 0; k < nops && ok; ++k) {
      if (!ops[k]->data) continue;
      ok = c.stride[k][w] == c.stride[k][d] * c.size[d];
    }
    if (ok) {
      c.size[w] *= c.size[d];
      for (int k = 0; k < nops; ++k) c.stride[k][w] = c.stride[k][d];
    } else {
      ++w;
      c.size[w] = c.size[d];
      for (int k = 0; k < nops; ++k) c.stride[k][w] = c.stride[k][d];
    }
  }
  c.ndim = c.ndim == 0 ? 0 : w + 1;
  return TSB_OK;
}

inline bool output_is_reduced(const Canon& c, int k) {
  for (int d = 0; d < c.ndim; ++d)
    if (c.stride[k][d] == 0) return true;
  return false;
}

inline int64_t align256(int64_t b) { return (b + 255) & ~int64_t(255); }

// Workspace bytes for the 2-D reduction kernel with TR-row tiles.
inline int64_t reduce_ws_bytes(const Canon& c, int n_in, const tsb_tensor* out, int n_out, int tr) {
  if (c.numel == 0) return 0;
  int64_t rows = 1, cols = 1;
  if (c.ndim == 1) cols = c.size[0];
  if (c.ndim == 2) {
    rows = c.size[0];
    cols = c.size[1];
  }
  const int64_t nrt = (rows + tr - 1) / tr, nct = (cols + kTC - 1) / kTC;
  int64_t total = 0;
  for (int o = 0; o < n_out; ++o) {
    if (!out[o].data) continue;
    const int k = n_in + o;
    if (!output_is_reduced(c, k)) continue;
    const int64_t s0 = c.ndim == 2 ? c.stride[k][0] : 0;
    const int64_t s1 = c.ndim >= 1 ? c.stride[k][c.ndim - 1] : 0;
    int64_t n;
    if (s0 != 0 && s1 == 0) n = nct * rows;
    else if (s0 == 0 && s1 != 0) n = nrt * cols;
    else n = nrt * nct;
    total += align256(n * (int64_t)sizeof(double));
  }
  return total;
}

// Resident CTAs per SM for one kernel instantiation, cached per device.
// `Tag` makes the cache (and the shared-memory opt-in) specific to the kernel:
// kernels of different functors can share a signature type.
template <class Tag, class K>
inline int occupancy_for(K kernel, int block, size_t smem, int dev) {
  static int cache[64];
  int* slot = dev >= 0 && dev < 64 ? &cache[dev] : nullptr;
  if (slot && *slot > 0) return *slot;
  // Opt in whenever dynamic shared memory is used: the default limit is
  // 48 KB minus the kernel's static shared memory.
  if (smem > 0) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, block, smem) != cudaSuccess || blocks < 1) {
    cudaGetLastError();
    blocks = 1;
  }
  if (slot) *slot = blocks;
  return blocks;
}

template <class Fn, typename TS>
struct MapTag {};
template <class Fn, typename TS>
struct ReduceTag {};
template <class Fn, typename TS, int PASS>
struct SweepTag {};

inline int32_t check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(TSB_ERR_LAUNCH, "%s: %s", what, cudaGetErrorString(e));
  return TSB_OK;
}

template <class Fn, typename TS>
int32_t launch_map(const MapParams<Fn::NIN, Fn::NOUT>& p, cudaStream_t stream, int dev, const DeviceInfo* info) {
  using S = typename MapTile<Fn>::S;
  constexpr size_t smem = Fn::R > 1 ? S::SMEM : 0;
  const int occ = occupancy_for<MapTag<Fn, TS>>(map_kernel<Fn, TS>, kBlock, smem, dev);
  const int64_t ntiles = (p.numel + S::TILE - 1) / S::TILE;
  const int64_t grid = std::min<int64_t>(ntiles, (int64_t)info->sm_count * occ);
  map_kernel<Fn, TS><<<(unsigned)grid, kBlock, smem, stream>>>(p);
  count_launches(1);
  return check_launch("map kernel launch");
}

template <int NIN, int NOUT>
inline int32_t fill_reduce_params(const Canon& c, const tsb_tensor* in, const tsb_tensor* out, uint32_t mask, void* ws,
                                  int64_t ws_bytes, int tr, Reduce2DParams<NIN, NOUT>& p);

template <class Fn, typename TS>
int32_t launch_reduce(const Canon& c, const tsb_tensor* in, const tsb_tensor* out, uint32_t mask, void* ws,
                      int64_t ws_bytes, cudaStream_t stream, int dev, const DeviceInfo* info) {
  Reduce2DParams<Fn::NIN, Fn::NOUT> p;
  const int32_t fst = fill_reduce_params(c, in, out, mask, ws, ws_bytes, ReduceTile<Fn>::TR, p);
  if (fst) return fst;
  constexpr size_t smem = ReduceStage<Fn>::SMEM;
  const int occ = occupancy_for<ReduceTag<Fn, TS>>(reduce2d_kernel<Fn, TS>, kBlock, smem, dev);
  const int64_t ntiles = p.n_row_tiles * p.n_col_tiles;
  const int64_t grid = std::min<int64_t>(ntiles, (int64_t)info->sm_count * occ);
  reduce2d_kernel<Fn, TS><<<(unsigned)grid, kBlock, smem, stream>>>(p);
  count_launches(1);
  int32_t st = check_launch("reduce kernel launch");
  if (st) return st;
  for (int o = 0; o < Fn::NOUT; ++o) {
    if (!(p.out_mask & (1u << o))) continue;
    const int kind = p.out_kind[o];
    if (kind == kOutRow) {
      launch_finalize<TS>(p.ws[o], p.rows, p.n_col_tiles, p.rows, p.out_ptr[o], p.out_s0[o], stream);
    } else if (kind == kOutCol) {
      launch_finalize<TS>(p.ws[o], p.cols, p.n_row_tiles, p.cols, p.out_ptr[o], p.out_s1[o], stream);
    } else if (kind == kOutAll) {
      finalize_all_kernel<TS><<<1, kBlock, 0, stream>>>(p.ws[o], ntiles, p.out_ptr[o]);
      count_launches(1);
    } else {
      continue;
    }
    st = check_launch("finalize kernel launch");
    if (st) return st;
  }
  return TSB_OK;
}

// Sweep layout: input ia constant along one dimension and varying along the
// other, input ix the reverse.  Sets `transpose` when ia varies along the
// columns (the problem is then swept with rows and columns exchanged).
inline bool sweep_layout(const Canon& c, int ia, int ix, bool& transpose) {
  if (c.ndim != 2) return false;
  const int64_t a0 = c.stride[ia][0], a1 = c.stride[ia][1], x0 = c.stride[ix][0], x1 = c.stride[ix][1];
  if (a0 != 0 && a1 == 0 && x0 == 0 && x1 != 0) transpose = false;
  else if (a0 == 0 && a1 != 0 && x0 != 0 && x1 == 0) transpose = true;
  else return false;
  return c.size[transpose ? 1 : 0] <= kSweepMaxRows;
}

// Functors whose reducing pass may run through the streaming 2-D kernel
// (stream2d.cuh): `static constexpr bool STREAM2D = true`.
template <class Fn, class = void>
struct Stream2DOptIn {
  static constexpr bool value = false;
};
template <class Fn>
struct Stream2DOptIn<Fn, decltype((void)Fn::STREAM2D, void())> {
  static constexpr bool value = Fn::STREAM2D;
};

// Streaming 2-D reduction; defined in stream2d.cuh, which the units of
// functors with STREAM2D include.  Returns TSB_ERR_LAYOUT without launching
// when the layout or the workspace does not suit it.
template <class Fn, typename TS>
int32_t launch_stream2d(const Canon& c, const tsb_tensor* in, const tsb_tensor* out, uint32_t mask, void* ws,
                        int64_t ws_bytes, cudaStream_t stream);

// Runs Fn through the row-sorted sweep; defined in sweep.cuh, which the
// units of functors with SWEEP include.  Returns TSB_ERR_WORKSPACE without
// launching when `ws` is too small for the partial sums and the sweep's
// scratch, so that the caller can fall back to the tile kernel.
template <class Fn, typename TS>
int32_t launch_sweep(const Canon& c, bool transpose, const tsb_tensor* out, uint32_t mask, const tsb_tensor* in,
                     void* ws, int64_t ws_bytes, cudaStream_t stream, int dev, const DeviceInfo* info);

template <int NIN, int NOUT>
inline void fill_map_params(const Canon& c, const tsb_tensor* in, const tsb_tensor* out, uint32_t mask,
                            MapParams<NIN, NOUT>& p) {
  p.ndim = c.ndim == 0 ? 1 : c.ndim;
  p.numel = c.numel;
  for (int d = 0; d < kMaxDims; ++d) p.size[d] = (d < c.ndim) ? c.size[d] : 1;
  bool dense = c.ndim <= 1;
  for (int k = 0; k < NIN + NOUT; ++k) {
    Operand& op = k < NIN ? p.in[k] : p.out[k - NIN];
    op.ptr = static_cast<char*>(k < NIN ? in[k].data : out[k - NIN].data);
    for (int d = 0; d < kMaxDims; ++d) op.stride[d] = (d < c.ndim) ? c.stride[k][d] : 0;
    const bool active = k < NIN || (mask & (1u << (k - NIN)));
    if (active && c.ndim == 1 && c.stride[k][0] != 1) dense = false;
  }
  p.dense = dense ? 1 : 0;
  p.out_mask = mask;
}

template <int NIN, int NOUT>
inline int32_t fill_reduce_params(const Canon& c, const tsb_tensor* in, const tsb_tensor* out, uint32_t mask,
                                  void* ws, int64_t ws_bytes, int tr, Reduce2DParams<NIN, NOUT>& p) {
  const int TR = tr;
  if (c.ndim > 2)
    return set_error(TSB_ERR_LAYOUT,
                     "reduced outputs need an iteration space that coalesces to at most 2 dims (got %d)", c.ndim);
  p.rows = c.ndim == 2 ? c.size[0] : 1;
  p.cols = c.ndim >= 1 ? c.size[c.ndim - 1] : 1;
  p.n_row_tiles = (p.rows + TR - 1) / TR;
  p.n_col_tiles = (p.cols + kTC - 1) / kTC;
  p.out_mask = mask;
  for (int k = 0; k < NIN; ++k) {
    p.in_ptr[k] = static_cast<char*>(in[k].data);
    p.in_s0[k] = c.ndim == 2 ? c.stride[k][0] : 0;
    p.in_s1[k] = c.ndim >= 1 ? c.stride[k][c.ndim - 1] : 0;
  }
  const int64_t need = reduce_ws_bytes(c, NIN, out, NOUT, TR);
  if (need > 0 && (!ws || ws_bytes < need))
    return set_error(TSB_ERR_WORKSPACE, "workspace of %lld bytes required, %lld given", (long long)need,
                     (long long)ws_bytes);
  if (need > 0 && ((uintptr_t)ws % 256) != 0) return set_error(TSB_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  char* wp = static_cast<char*>(ws);
  for (int o = 0; o < NOUT; ++o) {
    const int k = NIN + o;
    p.out_ptr[o] = static_cast<char*>(out[o].data);
    p.ws[o] = nullptr;
    p.out_kind[o] = kOutNone;
    p.out_s0[o] = p.out_s1[o] = 0;
    if (!(mask & (1u << o))) continue;
    const int64_t s0 = c.ndim == 2 ? c.stride[k][0] : 0;
    const int64_t s1 = c.ndim >= 1 ? c.stride[k][c.ndim - 1] : 0;
    p.out_s0[o] = s0;
    p.out_s1[o] = s1;
    int kind;
    int64_t n = 0;
    if (c.ndim == 2) {
      if (s0 != 0 && s1 != 0) kind = kOutFull;
      else if (s0 != 0) kind = kOutRow;
      else if (s1 != 0) kind = kOutCol;
      else kind = kOutAll;
    } else {
      kind = (s1 != 0) ? kOutFull : kOutAll;
    }
    if (kind == kOutRow) n = p.n_col_tiles * p.rows;
    if (kind == kOutCol) n = p.n_row_tiles * p.cols;
    if (kind == kOutAll) n = p.n_row_tiles * p.n_col_tiles;
    p.out_kind[o] = kind;
    if (n > 0) {
      p.ws[o] = reinterpret_cast<double*>(wp);
      wp += align256(n * (int64_t)sizeof(double));
    }
  }
  return TSB_OK;
}

// Generic entry point body.  F<double> is the FP64 functor, F<float> the
// mixed one; both have the same NIN / NOUT.
template <template <typename> class F>
int32_t run_op(const tsb_tensor* in, int32_t n_in, const tsb_tensor* out, int32_t n_out, int32_t precision, void* ws,
               int64_t ws_bytes, void* stream_ptr) {
  using FD = F<double>;
  using FF = F<float>;
  constexpr int NIN = FD::NIN, NOUT = FD::NOUT;
  static_assert(FF::NIN == NIN && FF::NOUT == NOUT, "functor arity mismatch");
  Canon c;
  int32_t dtype = 0;
  int32_t st = canonicalize(in, n_in, out, n_out, NIN, NOUT, c, dtype);
  if (st) return st;
  if (precision != TSB_PRECISION_AUTO && precision != TSB_PRECISION_FP64)
    return set_error(TSB_ERR_ARGUMENT, "unknown precision mode %d", precision);
  if (dtype == TSB_C64 || dtype == TSB_C128)
    return set_error(TSB_ERR_DTYPE, "this entry point takes real dtypes only");
  uint32_t mask = 0;
  for (int o = 0; o < NOUT; ++o)
    if (out[o].data) mask |= 1u << o;
  if (c.numel == 0 || mask == 0) return TSB_OK;
  int dev = 0;
  const DeviceInfo* info = nullptr;
  st = current_device(&dev, &info);
  if (st) return st;
  bool reduced = false;
  for (int o = 0; o < NOUT; ++o)
    if ((mask & (1u << o)) && output_is_reduced(c, NIN + o)) reduced = true;
  cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);
  const bool use64 = precision == TSB_PRECISION_FP64;
  if constexpr (HasAux<FD>::value && SweepOptIn<FD>::value) {
    // (R, 1) x (1, C) grids (or the transpose) with a workspace: the
    // row-sorted sweep.  Without room for its scratch, the tile kernel below.
    bool tr = false;
    if (ws && sweep_layout(c, FD::AUX_IN0, FD::AUX_IN1, tr)) {
      int32_t sw = TSB_ERR_DTYPE;
      switch (dtype) {
        case TSB_F64: sw = launch_sweep<FD, double>(c, tr, out, mask, in, ws, ws_bytes, s, dev, info); break;
        case TSB_F32:
          sw = use64 ? launch_sweep<FD, float>(c, tr, out, mask, in, ws, ws_bytes, s, dev, info)
                     : launch_sweep<FF, float>(c, tr, out, mask, in, ws, ws_bytes, s, dev, info);
          break;
        case TSB_F16: sw = launch_sweep<FF, __half>(c, tr, out, mask, in, ws, ws_bytes, s, dev, info); break;
        case TSB_BF16: sw = launch_sweep<FF, __nv_bfloat16>(c, tr, out, mask, in, ws, ws_bytes, s, dev, info); break;
      }
      if (sw != TSB_ERR_WORKSPACE) return sw;
    }
  }
  if constexpr (HasAux<FD>::value) {
    // A 2-D grid on which an input with per-row/column tables is broadcast
    // runs through the tiled 2-D kernel (every output full), which builds the
    // tables once per tile row / column.
    if (!reduced && c.ndim == 2) {
      const int ka = FD::AUX_IN0, kb = FD::AUX_IN1;
      const bool bcast = c.stride[ka][0] == 0 || c.stride[ka][1] == 0 || c.stride[kb][0] == 0 || c.stride[kb][1] == 0;
      if (bcast) {
        switch (dtype) {
          case TSB_F64: return launch_reduce<FD, double>(c, in, out, mask, nullptr, 0, s, dev, info);
          case TSB_F32:
            return use64 ? launch_reduce<FD, float>(c, in, out, mask, nullptr, 0, s, dev, info)
                         : launch_reduce<FF, float>(c, in, out, mask, nullptr, 0, s, dev, info);
          case TSB_F16: return launch_reduce<FF, __half>(c, in, out, mask, nullptr, 0, s, dev, info);
          case TSB_BF16: return launch_reduce<FF, __nv_bfloat16>(c, in, out, mask, nullptr, 0, s, dev, info);
        }
        return set_error(TSB_ERR_DTYPE, "unsupported dtype");
      }
    }
  }
  if (!reduced) {
    MapParams<NIN, NOUT> p;
    fill_map_params(c, in, out, mask, p);
    switch (dtype) {
      case TSB_F64: return launch_map<FD, double>(p, s, dev, info);
      case TSB_F32: return use64 ? launch_map<FD, float>(p, s, dev, info) : launch_map<FF, float>(p, s, dev, info);
      case TSB_F16: return launch_map<FF, __half>(p, s, dev, info);
      case TSB_BF16: return launch_map<FF, __nv_bfloat16>(p, s, dev, info);
    }
    return set_error(TSB_ERR_DTYPE, "unsupported dtype");
  }
  if constexpr (FD::REDUCE) {
    if constexpr (Stream2DOptIn<FD>::value) {
      int32_t sr = TSB_ERR_LAYOUT;
      switch (dtype) {
        case TSB_F64: sr = launch_stream2d<FD, double>(c, in, out, mask, ws, ws_bytes, s); break;
        case TSB_F32: sr = launch_stream2d<FF, float>(c, in, out, mask, ws, ws_bytes, s); break;
        case TSB_F16: sr = launch_stream2d<FF, __half>(c, in, out, mask, ws, ws_bytes, s); break;
        case TSB_BF16: sr = launch_stream2d<FF, __nv_bfloat16>(c, in, out, mask, ws, ws_bytes, s); break;
      }
      if (sr != TSB_ERR_LAYOUT) return sr;
    }
    switch (dtype) {
      case TSB_F64: return launch_reduce<FD, double>(c, in, out, mask, ws, ws_bytes, s, dev, info);
      case TSB_F32:
        return use64 ? launch_reduce<FD, float>(c, in, out, mask, ws, ws_bytes, s, dev, info)
                     : launch_reduce<FF, float>(c, in, out, mask, ws, ws_bytes, s, dev, info);
      case TSB_F16: return launch_reduce<FF, __half>(c, in, out, mask, ws, ws_bytes, s, dev, info);
      case TSB_BF16: return launch_reduce<FF, __nv_bfloat16>(c, in, out, mask, ws, ws_bytes, s, dev, info);
    }
    return set_error(TSB_ERR_DTYPE, "unsupported dtype");
  } else {
    return set_error(TSB_ERR_LAYOUT, "this entry point does not produce reduced outputs");
  }
}

// Entry point body for complex64 / complex128 data: the map kernel over a
// complex128 functor, no reduced outputs.
template <class CF>
int32_t run_complex(const tsb_tensor* in, int32_t n_in, const tsb_tensor* out, int32_t n_out, int32_t precision,
                    void* stream_ptr) {
  constexpr int NIN = CF::NIN, NOUT = CF::NOUT;
  Canon c;
  int32_t dtype = 0;
  int32_t st = canonicalize(in, n_in, out, n_out, NIN, NOUT, c, dtype);
  if (st) return st;
  if (precision != TSB_PRECISION_AUTO && precision != TSB_PRECISION_FP64)
    return set_error(TSB_ERR_ARGUMENT, "unknown precision mode %d", precision);
  uint32_t mask = 0;
  for (int o = 0; o < NOUT; ++o)
    if (out[o].data) mask |= 1u << o;
  if (c.numel == 0 || mask == 0) return TSB_OK;
  for (int o = 0; o < NOUT; ++o)
    if ((mask & (1u << o)) && output_is_reduced(c, NIN + o))
      return set_error(TSB_ERR_LAYOUT, "complex entry points do not reduce outputs");
  int dev = 0;
  const DeviceInfo* info = nullptr;
  st = current_device(&dev, &info);
  if (st) return st;
  MapParams<NIN, NOUT> p;
  fill_map_params(c, in, out, mask, p);
  cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);
  switch (dtype) {
    case TSB_C64: return launch_map<CF, cuda::std::complex<float>>(p, s, dev, info);
    case TSB_C128: return launch_map<CF, cuda::std::complex<double>>(p, s, dev, info);
  }
  return set_error(TSB_ERR_DTYPE, "unsupported dtype");
}

}  // namespace tsb

// Defines one C-ABI entry point that forwards to run_op<Functor>.
#define TSB_DEFINE_OP(cname, Functor)                                                                  \
  extern "C" TSB_OP_SIGNATURE(cname) {                                                                 \
    return tsb::run_op<Functor>(in, n_in, out, n_out, precision, workspace, workspace_bytes, stream); \
  }

// An entry point that also takes complex64 / complex128 data (run_complex
// with CFunctor, a complex128 functor).
#define TSB_DEFINE_OP_C(cname, Functor, CFunctor)                                                         \
  extern "C" TSB_OP_SIGNATURE(cname) {                                                                   \
    if (n_in > 0 && in && (in[0].dtype == TSB_C64 || in[0].dtype == TSB_C128))                           \
      return tsb::run_complex<CFunctor>(in, n_in, out, n_out, precision, stream);                        \
    return tsb::run_op<Functor>(in, n_in, out, n_out, precision, workspace, workspace_bytes, stream);   \
  }
