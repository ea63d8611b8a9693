// Elementwise map kernels for the special functions.
//
// One kernel template serves every (function, pass): a functor `Fn` supplies
//   using T;                       compute type (double = FP64 kernels,
//                                  float = mixed FP32 kernels)
//   static constexpr int NIN, NOUT, R;
//   __device__ static int  classify(const T* in);              (R > 1 only)
//   __device__ static void eval(int region, const T* in, T* out, uint32_t mask);
//
// When R > 1 each CTA works on a tile of TILE elements in four phases:
//   1. coalesced load of the tile's inputs (strided/broadcast gather through
//      the operand strides, or a dense fast path), region id per element;
//   2. compaction: per-warp __match_any_sync groups lanes with equal region,
//      one shared-memory atomic per group reserves slots, so the tile's local
//      indices end up bucketed by region in shared memory;
//   3. evaluation: consecutive threads take consecutive slots, so every warp
//      runs a single region's code path except at bucket boundaries;
//   4. results go back through shared memory and leave as coalesced stores.
// R == 1 functors skip the shared-memory staging.
//
// The 2-D variant (reduce2d_kernel) tiles an R x C iteration space in
// TR x 32 blocks and sums outputs whose stride is zero along a dimension:
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
constexpr int kBlock = 256;

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

template <class Fn>
struct TileShape {
  static constexpr int NBUF = Fn::NIN > Fn::NOUT ? Fn::NIN : Fn::NOUT;
  static constexpr int EPT = 4;
  static constexpr int TILE = kBlock * EPT;  // 1024 elements
  // Dynamic shared memory: staging buffer + region list + region ids.
  static constexpr size_t SMEM = (size_t)NBUF * TILE * sizeof(typename Fn::T) + TILE * sizeof(uint16_t) + TILE;
};

template <class Fn>
__device__ __forceinline__ void carve_smem(unsigned char* base, typename Fn::T*& buf, uint16_t*& list,
                                           uint8_t*& reg) {
  using T = typename Fn::T;
  buf = reinterpret_cast<T*>(base);
  list = reinterpret_cast<uint16_t*>(buf + TileShape<Fn>::NBUF * TileShape<Fn>::TILE);
  reg = reinterpret_cast<uint8_t*>(list + TileShape<Fn>::TILE);
}

// Bucket the tile's local indices by region.  `reg[k]` is the region of the
// element at local index k*kBlock + tid, or R (not valid).  On return
// s_list[0..count) holds local indices grouped by region, and s_reg[li] the
// region of local index li.
template <int R, int EPT>
__device__ __forceinline__ int compact_by_region(const int (&reg)[EPT], uint16_t* s_list,
                                                 uint8_t* s_reg, int* s_cnt) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  if (tid < R) s_cnt[tid] = 0;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < EPT; ++k) {
    const unsigned grp = __match_any_sync(0xffffffffu, reg[k]);
    const int leader = __ffs(grp) - 1;
    if (lane == leader && reg[k] < R) atomicAdd(&s_cnt[reg[k]], __popc(grp));
    s_reg[k * kBlock + tid] = static_cast<uint8_t>(reg[k]);
  }
  __syncthreads();
  // Exclusive scan over the R region counters (R is small).
  __shared__ int s_base[R + 1];
  if (tid == 0) {
    int acc = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      s_base[r] = acc;
      acc += s_cnt[r];
    }
    s_base[R] = acc;
  }
  __syncthreads();
  if (tid < R) s_cnt[tid] = s_base[tid];  // reuse as running cursor
  __syncthreads();
#pragma unroll
  for (int k = 0; k < EPT; ++k) {
    const unsigned grp = __match_any_sync(0xffffffffu, reg[k]);
    const int leader = __ffs(grp) - 1;
    int pos = 0;
    if (lane == leader && reg[k] < R) pos = atomicAdd(&s_cnt[reg[k]], __popc(grp));
    pos = __shfl_sync(0xffffffffu, pos, leader);
    if (reg[k] < R) s_list[pos + __popc(grp & lt_mask)] = static_cast<uint16_t>(k * kBlock + tid);
  }
  __syncthreads();
  return s_base[R];
}

template <class Fn, typename TS>
__global__ void __launch_bounds__(kBlock) map_kernel(const MapParams<Fn::NIN, Fn::NOUT> p) {
  using T = typename Fn::T;
  constexpr int NIN = Fn::NIN, NOUT = Fn::NOUT, R = Fn::R;
  constexpr int EPT = TileShape<Fn>::EPT, TILE = TileShape<Fn>::TILE, NBUF = TileShape<Fn>::NBUF;
  const int64_t ntiles = (p.numel + TILE - 1) / TILE;
  const int tid = threadIdx.x;

  if constexpr (R == 1) {
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
      T v[EPT][NIN];
#pragma unroll
      for (int k = 0; k < EPT; ++k) {
        const int64_t i = t * TILE + k * kBlock + tid;
        if (i < p.numel) load_element<Fn, TS>(p, i, v[k]);
      }
#pragma unroll
      for (int k = 0; k < EPT; ++k) {
        const int64_t i = t * TILE + k * kBlock + tid;
        if (i < p.numel) {
          T o[NOUT];
          Fn::eval(0, v[k], o, p.out_mask);
          store_element<Fn, TS>(p, i, o);
        }
      }
    }
  } else {
    extern __shared__ __align__(16) unsigned char s_dyn[];
    T* s_buf;
    uint16_t* s_list;
    uint8_t* s_reg;
    carve_smem<Fn>(s_dyn, s_buf, s_list, s_reg);
    __shared__ int s_cnt[R];
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const int64_t base = t * TILE;
      int reg[EPT];
#pragma unroll
      for (int k = 0; k < EPT; ++k) {
        const int li = k * kBlock + tid;
        const int64_t i = base + li;
        reg[k] = R;
        if (i < p.numel) {
          T v[NIN];
          load_element<Fn, TS>(p, i, v);
          reg[k] = Fn::classify(v);
#pragma unroll
          for (int q = 0; q < NIN; ++q) s_buf[q * TILE + li] = v[q];
        }
      }
      const int count = compact_by_region<R, EPT>(reg, s_list, s_reg, s_cnt);
      for (int j = tid; j < count; j += kBlock) {
        const int li = s_list[j];
        T v[NIN], o[NOUT];
#pragma unroll
        for (int q = 0; q < NIN; ++q) v[q] = s_buf[q * TILE + li];
        Fn::eval(s_reg[li], v, o, p.out_mask);
#pragma unroll
        for (int q = 0; q < NOUT; ++q) s_buf[q * TILE + li] = o[q];
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < EPT; ++k) {
        const int li = k * kBlock + tid;
        const int64_t i = base + li;
        if (i < p.numel) {
          T o[NOUT];
#pragma unroll
          for (int q = 0; q < NOUT; ++q) o[q] = s_buf[q * TILE + li];
          store_element<Fn, TS>(p, i, o);
        }
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------ 2-D reduction
constexpr int kTC = 32;  // tile columns (one warp wide)
constexpr int kTR = 1024 / kTC;  // tile rows (tiles hold 1024 elements)

template <class Fn>
struct Tile2D {
  static constexpr int TILE = TileShape<Fn>::TILE;
  static constexpr int TR = TILE / kTC;
  static_assert(TR == kTR, "2-D tiles are 32 x 32");
};

template <class Fn, typename TS>
__global__ void __launch_bounds__(kBlock) reduce2d_kernel(const Reduce2DParams<Fn::NIN, Fn::NOUT> p) {
  using T = typename Fn::T;
  constexpr int NIN = Fn::NIN, NOUT = Fn::NOUT, R = Fn::R;
  constexpr int EPT = TileShape<Fn>::EPT, TILE = TileShape<Fn>::TILE, NBUF = TileShape<Fn>::NBUF;
  constexpr int TR = Tile2D<Fn>::TR;
  constexpr int RR = R > 1 ? R : 1;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  T* s_buf;
  uint16_t* s_list;
  uint8_t* s_reg;
  carve_smem<Fn>(s_dyn, s_buf, s_list, s_reg);
  __shared__ int s_cnt[RR];
  __shared__ double s_red[kBlock / 32][kTC];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t ntiles = p.n_row_tiles * p.n_col_tiles;

  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t rt = t / p.n_col_tiles, ct = t % p.n_col_tiles;
    const int64_t r0 = rt * TR, c0 = ct * kTC;
    int reg[EPT];
#pragma unroll
    for (int k = 0; k < EPT; ++k) {
      const int li = k * kBlock + tid;
      const int64_t r = r0 + li / kTC, c = c0 + li % kTC;
      reg[k] = R;
      if (r < p.rows && c < p.cols) {
        T v[NIN];
#pragma unroll
        for (int q = 0; q < NIN; ++q)
          v[q] = load_as<TS, T>(p.in_ptr[q] + (r * p.in_s0[q] + c * p.in_s1[q]) * (int64_t)sizeof(TS));
        if constexpr (R > 1) reg[k] = Fn::classify(v);
        else reg[k] = 0;
#pragma unroll
        for (int q = 0; q < NIN; ++q) s_buf[q * TILE + li] = v[q];
      }
    }
    int count;
    if constexpr (R > 1) {
      count = compact_by_region<R, EPT>(reg, s_list, s_reg, s_cnt);
    } else {
      // No compaction: each thread evaluates its own elements in place.
      count = -1;
      __syncthreads();
    }
    if (count >= 0) {
      for (int j = tid; j < count; j += kBlock) {
        const int li = s_list[j];
        T v[NIN], o[NOUT];
#pragma unroll
        for (int q = 0; q < NIN; ++q) v[q] = s_buf[q * TILE + li];
        Fn::eval(s_reg[li], v, o, p.out_mask);
#pragma unroll
        for (int q = 0; q < NOUT; ++q) s_buf[q * TILE + li] = o[q];
      }
    } else {
#pragma unroll
      for (int k = 0; k < EPT; ++k) {
        const int li = k * kBlock + tid;
        if (reg[k] < R) {
          const int64_t r = r0 + li / kTC, c = c0 + li % kTC;
          if (r < p.rows && c < p.cols) {
            T v[NIN], o[NOUT];
#pragma unroll
            for (int q = 0; q < NIN; ++q) v[q] = s_buf[q * TILE + li];
            Fn::eval(0, v, o, p.out_mask);
#pragma unroll
            for (int q = 0; q < NOUT; ++q) s_buf[q * TILE + li] = o[q];
          }
        }
      }
    }
    __syncthreads();

    const int rows_here = (int)(p.rows - r0 < (int64_t)TR ? p.rows - r0 : (int64_t)TR);
    const int cols_here = (int)(p.cols - c0 < (int64_t)kTC ? p.cols - c0 : (int64_t)kTC);
#pragma unroll
    for (int o = 0; o < NOUT; ++o) {
      if (!(p.out_mask & (1u << o))) continue;
      const int kind = p.out_kind[o];
      if (kind == kOutFull) {
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
          const int li = k * kBlock + tid;
          const int lr = li / kTC, lc = li % kTC;
          if (lr < rows_here && lc < cols_here)
            store_as<TS>(p.out_ptr[o] + ((r0 + lr) * p.out_s0[o] + (c0 + lc) * p.out_s1[o]) * (int64_t)sizeof(TS),
                         s_buf[o * TILE + li]);
        }
      } else if (kind == kOutRow || kind == kOutAll) {
        // Row sums over this tile's columns: warp w takes rows w, w+8, ...
        // lane = column; fixed shuffle tree => deterministic.
        double tile_sum = 0.0;
        for (int lr = warp; lr < TR; lr += kBlock / 32) {
          double v = (lr < rows_here && lane < cols_here) ? (double)s_buf[o * TILE + lr * kTC + lane] : 0.0;
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
          if (kind == kOutRow) {
            if (lane == 0 && lr < rows_here) p.ws[o][ct * p.rows + r0 + lr] = v;
          } else {
            tile_sum += v;
          }
        }
        if (kind == kOutAll) {
          if (lane == 0) s_red[warp][0] = tile_sum;
          __syncthreads();
          if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < kBlock / 32; ++w) s += s_red[w][0];
            p.ws[o][t] = s;
          }
        }
      } else if (kind == kOutCol) {
        // Column sums over this tile's rows: warp w sums rows w, w+8, ...
        // per lane (= column), then warp partials are added in order.
        double v = 0.0;
        for (int lr = warp; lr < rows_here; lr += kBlock / 32) v += (double)s_buf[o * TILE + lr * kTC + lane];
        s_red[warp][lane] = v;
        __syncthreads();
        if (warp == 0) {
          double s = 0.0;
#pragma unroll
          for (int w = 0; w < kBlock / 32; ++w) s += s_red[w][lane];
          if (lane < cols_here) p.ws[o][rt * p.cols + c0 + lane] = s;
        }
      }
      __syncthreads();
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
