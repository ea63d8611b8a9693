// Elementwise map kernels for the special functions.
//
// One kernel template serves every (function, pass): a functor `Fn` supplies
//   using T;                       compute type (double = FP64 kernels,
//                                  float = mixed FP32 kernels)
//   static constexpr int NIN, NOUT, R;
//   __device__ static int  classify(const T* in);              (R > 1 only)
//   __device__ static void eval(int region, const T* in, T* out, uint32_t mask);
//
// When R > 1 each warp works on its own chunk of 256 elements (no CTA-wide
// barriers, so warps never wait for one another):
//   1. coalesced load of the chunk's inputs (strided/broadcast gather through
//      the operand strides, or a dense fast path) into a per-warp shared
//      memory slice, and a region id per element;
//   2. a ballot/popc prefix pass sorts the chunk's local indices by region
//      (deterministic order);
//   3. the warp evaluates the sorted list 32 at a time, so each round runs
//      one region's code path except at region boundaries;
//   4. results leave through the slice as coalesced stores.
// R == 1 functors skip the staging and evaluate straight from registers.
//
// The 2-D variant (reduce2d_kernel) tiles an R x C iteration space in
// 8 x 32 blocks and sums outputs whose stride is zero along a dimension:
// per-tile row/column partial sums in double land in a workspace and a
// second kernel adds the partials in tile order, so results are
// deterministic.  This is how backward kernels hand back gradients already
// reduced to the shape of a broadcast input.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "torchscience_b200.h"

namespace tsb {

constexpr int kMaxDims = TSB_MAX_DIMS;
constexpr int kBlock = 256;  // block size of the finalize kernels

struct Operand {
  char* ptr;
  int64_t stride[kMaxDims];  // element strides, row-major dims
};

template <int NIN, int NOUT>
struct MapParams {
  int32_t ndim;
  int32_t dense;  // 1: ndim == 1 and every operand has stride 1
  int64_t numel;
  int64_t size[kMaxDims];
  Operand in[NIN];
  Operand out[NOUT];
  uint32_t out_mask;  // bit o set: output o requested
};

// Output kinds of the 2-D reduction kernel.
enum OutKind : int32_t { kOutNone = 0, kOutFull = 1, kOutRow = 2, kOutCol = 3, kOutAll = 4 };

template <int NIN, int NOUT>
struct Reduce2DParams {
  int64_t rows, cols;
  int64_t n_row_tiles, n_col_tiles;
  char* in_ptr[NIN];
  int64_t in_s0[NIN], in_s1[NIN];
  char* out_ptr[NOUT];
  int64_t out_s0[NOUT], out_s1[NOUT];
  int32_t out_kind[NOUT];
  double* ws[NOUT];  // partial sums for reduced outputs
  uint32_t out_mask;
};

// ---------------------------------------------------------------- storage I/O
template <typename TS, typename T>
__device__ __forceinline__ T load_as(const char* p) {
  return static_cast<T>(__ldg(reinterpret_cast<const TS*>(p)));
}
template <>
__device__ __forceinline__ float load_as<__half, float>(const char* p) {
  return __half2float(*reinterpret_cast<const __half*>(p));
}
template <>
__device__ __forceinline__ float load_as<__nv_bfloat16, float>(const char* p) {
  return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(p));
}

template <typename TS, typename T>
__device__ __forceinline__ void store_as(char* p, T v) {
  *reinterpret_cast<TS*>(p) = static_cast<TS>(v);
}
template <>
__device__ __forceinline__ void store_as<__half, float>(char* p, float v) {
  *reinterpret_cast<__half*>(p) = __float2half_rn(v);
}
template <>
__device__ __forceinline__ void store_as<__nv_bfloat16, float>(char* p, float v) {
  *reinterpret_cast<__nv_bfloat16*>(p) = __float2bfloat16_rn(v);
}
template <>
__device__ __forceinline__ void store_as<__half, double>(char* p, double v) {
  *reinterpret_cast<__half*>(p) = __double2half(v);
}
template <>
__device__ __forceinline__ void store_as<__nv_bfloat16, double>(char* p, double v) {
  *reinterpret_cast<__nv_bfloat16*>(p) = __double2bfloat16(v);
}

// Element offsets of linear index i for every operand (row-major iteration).
template <int NIN, int NOUT>
__device__ __forceinline__ void linear_to_offsets(const MapParams<NIN, NOUT>& p, int64_t i,
                                                  int64_t (&oin)[NIN], int64_t (&oout)[NOUT]) {
#pragma unroll
  for (int k = 0; k < NIN; ++k) oin[k] = 0;
#pragma unroll
  for (int k = 0; k < NOUT; ++k) oout[k] = 0;
  if (p.numel <= 0xffffffffll) {
    uint32_t r = static_cast<uint32_t>(i);
    for (int d = p.ndim - 1; d >= 0; --d) {
      const uint32_t s = static_cast<uint32_t>(p.size[d]);
      const uint32_t c = r % s;
      r /= s;
#pragma unroll
      for (int k = 0; k < NIN; ++k) oin[k] += static_cast<int64_t>(c) * p.in[k].stride[d];
#pragma unroll
      for (int k = 0; k < NOUT; ++k) oout[k] += static_cast<int64_t>(c) * p.out[k].stride[d];
    }
  } else {
    int64_t r = i;
    for (int d = p.ndim - 1; d >= 0; --d) {
      const int64_t c = r % p.size[d];
      r /= p.size[d];
#pragma unroll
      for (int k = 0; k < NIN; ++k) oin[k] += c * p.in[k].stride[d];
#pragma unroll
      for (int k = 0; k < NOUT; ++k) oout[k] += c * p.out[k].stride[d];
    }
  }
}

template <class Fn, typename TS>
__device__ __forceinline__ void load_element(const MapParams<Fn::NIN, Fn::NOUT>& p, int64_t i,
                                             typename Fn::T (&v)[Fn::NIN]) {
  using T = typename Fn::T;
  if (p.dense) {
#pragma unroll
    for (int k = 0; k < Fn::NIN; ++k) v[k] = load_as<TS, T>(p.in[k].ptr + i * (int64_t)sizeof(TS));
  } else {
    int64_t oin[Fn::NIN], oout[Fn::NOUT];
    linear_to_offsets(p, i, oin, oout);
#pragma unroll
    for (int k = 0; k < Fn::NIN; ++k) v[k] = load_as<TS, T>(p.in[k].ptr + oin[k] * (int64_t)sizeof(TS));
  }
}

template <class Fn, typename TS>
__device__ __forceinline__ void store_element(const MapParams<Fn::NIN, Fn::NOUT>& p, int64_t i,
                                              const typename Fn::T (&v)[Fn::NOUT]) {
  if (p.dense) {
#pragma unroll
    for (int k = 0; k < Fn::NOUT; ++k)
      if (p.out_mask & (1u << k)) store_as<TS>(p.out[k].ptr + i * (int64_t)sizeof(TS), v[k]);
  } else {
    int64_t oin[Fn::NIN], oout[Fn::NOUT];
    linear_to_offsets(p, i, oin, oout);
#pragma unroll
    for (int k = 0; k < Fn::NOUT; ++k)
      if (p.out_mask & (1u << k)) store_as<TS>(p.out[k].ptr + oout[k] * (int64_t)sizeof(TS), v[k]);
  }
}

// ------------------------------------------------------------ warp chunks
// Every warp works on its own chunk of kChunk = 8 x 32 elements, independent
// of the other warps of its CTA (no block-wide barriers: a warp whose chunk
// holds long continued fractions does not hold up its neighbours).
constexpr int kEPT = 8;            // elements per lane per chunk
constexpr int kChunk = 32 * kEPT;  // 256
constexpr int kTC = 32;            // 2-D tile columns (one per lane)
constexpr int kTR = kEPT;          // 2-D tile rows

template <class Fn>
struct WarpStage {
  using T = typename Fn::T;
  static constexpr int NBUF = Fn::NIN > Fn::NOUT ? Fn::NIN : Fn::NOUT;
  // Per-warp shared memory: operand staging + region-sorted list + regions.
  static constexpr size_t PER_WARP = (size_t)NBUF * kChunk * sizeof(T) + 2 * kChunk;
  // Warps per CTA: at most 8, fewer when a warp's slice is large.
  static constexpr int WARPS = PER_WARP * 8 <= 64 * 1024 ? 8 : PER_WARP * 4 <= 64 * 1024 ? 4 : 2;
  static constexpr int BLOCK = 32 * WARPS;
  static constexpr size_t SMEM = Fn::R > 1 ? PER_WARP * WARPS : 0;
};

// Sorts the chunk's local indices by region with ballot prefix counts
// (deterministic order); returns the number of valid elements.  reg[k] is
// the region of local index k*32 + lane, or R for an invalid slot.
template <int R>
__device__ __forceinline__ int warp_sort_by_region(const int (&reg)[kEPT], uint8_t* list, uint8_t* regs) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  int count = 0;
#pragma unroll
  for (int k = 0; k < kEPT; ++k) regs[k * 32 + lane] = static_cast<uint8_t>(reg[k]);
#pragma unroll 1
  for (int r = 0; r < R; ++r) {
#pragma unroll
    for (int k = 0; k < kEPT; ++k) {
      const unsigned m = __ballot_sync(0xffffffffu, reg[k] == r);
      if (reg[k] == r) list[count + __popc(m & lt)] = static_cast<uint8_t>(k * 32 + lane);
      count += __popc(m);
    }
  }
  __syncwarp();
  return count;
}

// Evaluates the sorted chunk in place: inputs are read from, and outputs
// written to, the staging slots of each local index.
template <class Fn>
__device__ __forceinline__ void warp_eval_sorted(int count, typename Fn::T* buf, const uint8_t* list,
                                                 const uint8_t* regs, uint32_t mask) {
  using T = typename Fn::T;
  const int lane = threadIdx.x & 31;
  for (int j = lane; j < count; j += 32) {
    const int li = list[j];
    T v[Fn::NIN], o[Fn::NOUT];
#pragma unroll
    for (int q = 0; q < Fn::NIN; ++q) v[q] = buf[q * kChunk + li];
    Fn::eval(regs[li], v, o, mask);
#pragma unroll
    for (int q = 0; q < Fn::NOUT; ++q) buf[q * kChunk + li] = o[q];
  }
  __syncwarp();
}

template <class Fn>
__device__ __forceinline__ void warp_slice(unsigned char* base, typename Fn::T*& buf, uint8_t*& list,
                                           uint8_t*& regs) {
  using T = typename Fn::T;
  const int warp = threadIdx.x >> 5;
  unsigned char* w = base + warp * WarpStage<Fn>::PER_WARP;
  buf = reinterpret_cast<T*>(w);
  list = w + (size_t)WarpStage<Fn>::NBUF * kChunk * sizeof(T);
  regs = list + kChunk;
}

template <class Fn, typename TS>
__global__ void __launch_bounds__(256) map_kernel(const MapParams<Fn::NIN, Fn::NOUT> p) {
  using T = typename Fn::T;
  constexpr int NIN = Fn::NIN, NOUT = Fn::NOUT, R = Fn::R;
  const int lane = threadIdx.x & 31;
  const int64_t nchunks = (p.numel + kChunk - 1) / kChunk;
  const int64_t wid = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);

  if constexpr (R == 1) {
    for (int64_t c = wid; c < nchunks; c += nw) {
      const int64_t base = c * kChunk;
      T v[kEPT][NIN];
#pragma unroll
      for (int k = 0; k < kEPT; ++k) {
        const int64_t i = base + k * 32 + lane;
        if (i < p.numel) load_element<Fn, TS>(p, i, v[k]);
      }
#pragma unroll
      for (int k = 0; k < kEPT; ++k) {
        const int64_t i = base + k * 32 + lane;
        if (i < p.numel) {
          T o[NOUT];
          Fn::eval(0, v[k], o, p.out_mask);
          store_element<Fn, TS>(p, i, o);
        }
      }
    }
  } else {
    extern __shared__ __align__(16) unsigned char s_dyn[];
    T* buf;
    uint8_t *list, *regs;
    warp_slice<Fn>(s_dyn, buf, list, regs);
    for (int64_t c = wid; c < nchunks; c += nw) {
      const int64_t base = c * kChunk;
      int reg[kEPT];
#pragma unroll
      for (int k = 0; k < kEPT; ++k) {
        const int li = k * 32 + lane;
        const int64_t i = base + li;
        reg[k] = R;
        if (i < p.numel) {
          T v[NIN];
          load_element<Fn, TS>(p, i, v);
          reg[k] = Fn::classify(v);
#pragma unroll
          for (int q = 0; q < NIN; ++q) buf[q * kChunk + li] = v[q];
        }
      }
      __syncwarp();
      const int count = warp_sort_by_region<R>(reg, list, regs);
      warp_eval_sorted<Fn>(count, buf, list, regs, p.out_mask);
#pragma unroll
      for (int k = 0; k < kEPT; ++k) {
        const int li = k * 32 + lane;
        const int64_t i = base + li;
        if (i < p.numel) {
          T o[NOUT];
#pragma unroll
          for (int q = 0; q < NOUT; ++q) o[q] = buf[q * kChunk + li];
          store_element<Fn, TS>(p, i, o);
        }
      }
      __syncwarp();
    }
  }
}

// ------------------------------------------------------------ 2-D reduction
// Tiles of kTR rows x 32 columns, one per warp chunk: lane = column, the
// lane's kEPT elements are the tile's rows.  Row-reduced outputs take a
// shuffle tree per row, column-reduced outputs a fixed-order sum over the
// lane's rows; per-tile partials (double) go to the workspace.
template <class Fn, typename TS>
__global__ void __launch_bounds__(256) reduce2d_kernel(const Reduce2DParams<Fn::NIN, Fn::NOUT> p) {
  using T = typename Fn::T;
  constexpr int NIN = Fn::NIN, NOUT = Fn::NOUT, R = Fn::R;
  const int lane = threadIdx.x & 31;
  const int64_t ntiles = p.n_row_tiles * p.n_col_tiles;
  const int64_t wid = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  extern __shared__ __align__(16) unsigned char s_dyn[];
  T* buf = nullptr;
  uint8_t *list = nullptr, *regs = nullptr;
  if constexpr (R > 1) warp_slice<Fn>(s_dyn, buf, list, regs);

  for (int64_t t = wid; t < ntiles; t += nw) {
    const int64_t rt = t / p.n_col_tiles, ct = t % p.n_col_tiles;
    const int64_t r0 = rt * kTR, c = ct * kTC + lane;
    const bool col_ok = c < p.cols;
    T res[kEPT][NOUT];
    bool ok[kEPT];
#pragma unroll
    for (int k = 0; k < kEPT; ++k) ok[k] = col_ok && (r0 + k) < p.rows;

    if constexpr (R == 1) {
#pragma unroll
      for (int k = 0; k < kEPT; ++k) {
        if (ok[k]) {
          T v[NIN];
#pragma unroll
          for (int q = 0; q < NIN; ++q)
            v[q] = load_as<TS, T>(p.in_ptr[q] + ((r0 + k) * p.in_s0[q] + c * p.in_s1[q]) * (int64_t)sizeof(TS));
          Fn::eval(0, v, res[k], p.out_mask);
        } else {
#pragma unroll
          for (int q = 0; q < NOUT; ++q) res[k][q] = T(0);
        }
      }
    } else {
      int reg[kEPT];
#pragma unroll
      for (int k = 0; k < kEPT; ++k) {
        const int li = k * 32 + lane;
        reg[k] = R;
        if (ok[k]) {
          T v[NIN];
#pragma unroll
          for (int q = 0; q < NIN; ++q)
            v[q] = load_as<TS, T>(p.in_ptr[q] + ((r0 + k) * p.in_s0[q] + c * p.in_s1[q]) * (int64_t)sizeof(TS));
          reg[k] = Fn::classify(v);
#pragma unroll
          for (int q = 0; q < NIN; ++q) buf[q * kChunk + li] = v[q];
        }
      }
      __syncwarp();
      const int count = warp_sort_by_region<R>(reg, list, regs);
      warp_eval_sorted<Fn>(count, buf, list, regs, p.out_mask);
#pragma unroll
      for (int k = 0; k < kEPT; ++k)
#pragma unroll
        for (int q = 0; q < NOUT; ++q) res[k][q] = ok[k] ? buf[q * kChunk + k * 32 + lane] : T(0);
      __syncwarp();
    }

#pragma unroll
    for (int o = 0; o < NOUT; ++o) {
      if (!(p.out_mask & (1u << o))) continue;
      const int kind = p.out_kind[o];
      if (kind == kOutFull) {
#pragma unroll
        for (int k = 0; k < kEPT; ++k)
          if (ok[k])
            store_as<TS>(p.out_ptr[o] + ((r0 + k) * p.out_s0[o] + c * p.out_s1[o]) * (int64_t)sizeof(TS), res[k][o]);
      } else if (kind == kOutRow) {
#pragma unroll
        for (int k = 0; k < kEPT; ++k) {
          double v = (double)res[k][o];
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
          if (lane == 0 && r0 + k < p.rows) p.ws[o][ct * p.rows + r0 + k] = v;
        }
      } else if (kind == kOutCol) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < kEPT; ++k) v += (double)res[k][o];
        if (col_ok) p.ws[o][rt * p.cols + c] = v;
      } else if (kind == kOutAll) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < kEPT; ++k) v += (double)res[k][o];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) p.ws[o][t] = v;
      }
    }
  }
}

// Adds the per-tile partials of one reduced output in tile order.
template <typename TS>
__global__ void __launch_bounds__(kBlock) finalize_kernel(const double* ws, int64_t n_out, int64_t n_parts,
                                                          int64_t part_stride, char* out, int64_t out_stride) {
  const int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x;
  if (i >= n_out) return;
  double s = 0.0;
  for (int64_t k = 0; k < n_parts; ++k) s += ws[k * part_stride + i];
  store_as<TS>(out + i * out_stride * (int64_t)sizeof(TS), s);
}

// Deterministic sum of n partials (single CTA, fixed tree) into out[0].
template <typename TS>
__global__ void __launch_bounds__(kBlock) finalize_all_kernel(const double* ws, int64_t n_parts, char* out) {
  __shared__ double s[kBlock];
  double v = 0.0;
  for (int64_t k = threadIdx.x; k < n_parts; k += kBlock) v += ws[k];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int w = kBlock / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) store_as<TS>(out, s[0]);
}

}  // namespace tsb
