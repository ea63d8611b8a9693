// Elementwise map kernels for the special functions.
//
// One kernel template serves every (function, pass): a functor `Fn` supplies
//   using T;                       compute type (double = FP64 kernels,
//                                  float = mixed FP32 kernels)
//   static constexpr int NIN, NOUT, R;
//   __device__ static int  classify(const T* in);              (R > 1 only)
//   __device__ static void eval(int region, const T* in, T* out, uint32_t mask);
//
// When R > 1 each CTA works on a tile of up to 2048 elements in four phases:
//   1. coalesced load of the tile's inputs (strided/broadcast gather through
//      the operand strides, or a dense fast path), region id per element;
//   2. compaction: per-warp __match_any_sync groups lanes with equal region,
//      one shared-memory atomic per group reserves slots, so the tile's local
//      indices end up bucketed by region in shared memory;
//   3. evaluation: consecutive threads take consecutive slots, so every warp
//      runs a single region's code path except at bucket boundaries, and the
//      32-slot groups go round-robin to the warps so their loads balance;
//   4. results go back through shared memory and leave as coalesced stores.
// R == 1 functors skip the shared-memory staging.  Regions are both the
// evaluation method and, for iterative methods, a bucket of the expected
// iteration count, so warps run loops of similar length.
//
// The 2-D variant (reduce2d_kernel) tiles an R x C iteration space in
// 32 x 32 blocks and sums outputs whose stride is zero along a dimension:
// per-tile row/column partial sums in double land in a workspace and a
// second kernel adds the partials in tile order, so results are
// deterministic.  This is how backward kernels hand back gradients already
// reduced to the shape of a broadcast input.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cuda/std/complex>

#include <type_traits>

#include "torchscience_b200.h"
#include "unconverged.cuh"

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

// Complex storage (interleaved real, imaginary) with complex128 arithmetic.
template <>
__device__ __forceinline__ cuda::std::complex<double> load_as<cuda::std::complex<float>, cuda::std::complex<double>>(
    const char* p) {
  const float2 v = __ldg(reinterpret_cast<const float2*>(p));
  return cuda::std::complex<double>(v.x, v.y);
}
template <>
__device__ __forceinline__ cuda::std::complex<double> load_as<cuda::std::complex<double>, cuda::std::complex<double>>(
    const char* p) {
  const double2 v = __ldg(reinterpret_cast<const double2*>(p));
  return cuda::std::complex<double>(v.x, v.y);
}
template <>
__device__ __forceinline__ void store_as<cuda::std::complex<float>, cuda::std::complex<double>>(
    char* p, cuda::std::complex<double> v) {
  *reinterpret_cast<float2*>(p) = make_float2((float)v.real(), (float)v.imag());
}
template <>
__device__ __forceinline__ void store_as<cuda::std::complex<double>, cuda::std::complex<double>>(
    char* p, cuda::std::complex<double> v) {
  *reinterpret_cast<double2*>(p) = make_double2(v.real(), v.imag());
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

// ------------------------------------------------------------ CTA tiles
// Map kernels stage tiles of up to 2048 elements (1024 when the operands
// need more shared memory); the 2-D reduction uses 32 x 32 tiles.
constexpr int kTC = 32;     // 2-D tile columns (one per lane)
constexpr int kTRMin = 32;  // smallest 2-D tile height (sizes the generic workspace query)

template <class Fn, int TILE_, int NBUF_ = (Fn::NIN > Fn::NOUT ? Fn::NIN : Fn::NOUT)>
struct Stage {
  using T = typename Fn::T;
  static constexpr int NBUF = NBUF_;
  static constexpr int TILE = TILE_;
  static constexpr int EPT = TILE / kBlock;
  // operand staging + region-sorted list (uint16) + region ids (uint8)
  static constexpr size_t SMEM = (size_t)NBUF * TILE * sizeof(T) + TILE * sizeof(uint16_t) + TILE;
};

template <class Fn>
struct MapTile {
  static constexpr int BIG = Stage<Fn, 2048>::SMEM <= 64 * 1024 ? 2048 : 1024;
  using S = Stage<Fn, (Fn::R > 1 ? BIG : 1024)>;
};

template <class S>
__device__ __forceinline__ void carve(unsigned char* base, typename S::T*& buf, uint16_t*& list, uint8_t*& regs) {
  using T = typename S::T;
  buf = reinterpret_cast<T*>(base);
  list = reinterpret_cast<uint16_t*>(buf + (size_t)S::NBUF * S::TILE);
  regs = reinterpret_cast<uint8_t*>(list + S::TILE);
}

// Optional per-input tables (functors that define NAUX0): quantities of one
// input alone (e.g. lnΓ(a), ψ(a), ln x) that a 2-D tile computes once per
// row or column into shared memory when that input is constant along the
// other dimension.  Such a functor provides
//   AUX_IN0, AUX_IN1          the two inputs with tables,
//   NAUX0, NAUX1              doubles per table entry,
//   make_aux0(v, o), make_aux1(v, o),
//   classify(in, aux0, aux1), eval(r, in, out, mask, aux0, aux1)
// where a null table pointer means "compute the quantity here".
template <class Fn, class = void>
struct HasAux {
  static constexpr bool value = false;
  static constexpr int N0 = 1, N1 = 1;
};
template <class Fn>
struct HasAux<Fn, decltype((void)Fn::NAUX0, void())> {
  static constexpr bool value = true;
  static constexpr int N0 = Fn::NAUX0, N1 = Fn::NAUX1;
};

// Resident CTAs per SM the register allocation must allow (functors may set
// MIN_BLOCKS; the default leaves registers unconstrained).
template <class Fn, class = void>
struct MinBlocks {
  static constexpr int value = 1;
};
template <class Fn>
struct MinBlocks<Fn, decltype((void)Fn::MIN_BLOCKS, void())> {
  static constexpr int value = Fn::MIN_BLOCKS;
};

// Rows of a 2-D tile: a functor's TILE_ROWS (32 or 64) if it sets one, else
// 64 when the staging fits in 64 KB and 32 otherwise.
template <class Fn, class = void>
struct TileRows {
  static constexpr int value = 0;
};
template <class Fn>
struct TileRows<Fn, decltype((void)Fn::TILE_ROWS, void())> {
  static constexpr int value = Fn::TILE_ROWS;
};

template <class Fn, class = void>
struct HasAuxIdx {
  static constexpr int i0 = -1, i1 = -1;
};
template <class Fn>
struct HasAuxIdx<Fn, decltype((void)Fn::NAUX0, void())> {
  static constexpr int i0 = Fn::AUX_IN0, i1 = Fn::AUX_IN1;
};

// Table modes: 0 none (computed per element), 1 one entry per tile row,
// 2 one entry per tile column.
__device__ __forceinline__ int aux_mode(int64_t s0, int64_t s1) { return s1 == 0 ? 1 : (s0 == 0 ? 2 : 0); }
template <int N>
__device__ __forceinline__ const double* aux_at(const double* tab, int mode, int li) {
  return mode == 1 ? tab + (li / 32) * N : (mode == 2 ? tab + (li % 32) * N : nullptr);
}

// Buckets the tile's local indices by region.  reg[k] is the region of
// local index k*kBlock + tid, or R for an invalid slot.  On return
// list[0..count) holds the valid local indices grouped by region and
// regs[li] the region of li.  (Order inside a region depends on atomic
// order; results do not, each element being evaluated independently.)
template <int R, int EPT>
__device__ __forceinline__ int cta_sort_by_region(const int (&reg)[EPT], uint16_t* list, uint8_t* regs, int* s_cnt,
                                                  int* s_base, int* s_next) {
  const int tid = threadIdx.x, lane = tid & 31;
  const unsigned lt = (1u << lane) - 1u;
  if (tid < R) s_cnt[tid] = 0;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < EPT; ++k) {
    const unsigned grp = __match_any_sync(0xffffffffu, reg[k]);
    if (lane == __ffs(grp) - 1 && reg[k] < R) atomicAdd(&s_cnt[reg[k]], __popc(grp));
    regs[k * kBlock + tid] = static_cast<uint8_t>(reg[k]);
  }
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      s_base[r] = acc;
      acc += s_cnt[r];
    }
    s_base[R] = acc;
    *s_next = 0;
  }
  __syncthreads();
  if (tid < R) s_cnt[tid] = s_base[tid];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < EPT; ++k) {
    const unsigned grp = __match_any_sync(0xffffffffu, reg[k]);
    const int leader = __ffs(grp) - 1;
    int pos = 0;
    if (lane == leader && reg[k] < R) pos = atomicAdd(&s_cnt[reg[k]], __popc(grp));
    pos = __shfl_sync(0xffffffffu, pos, leader);
    if (reg[k] < R) list[pos + __popc(grp & lt)] = static_cast<uint16_t>(k * kBlock + tid);
  }
  __syncthreads();
  return s_base[R];
}

// Functors whose fast evaluation may decline an element (RESCUE = true):
//   __device__ static bool eval_first(int region, const T* in, T* out, uint32_t mask)
//     evaluates and returns true, or returns false (out untouched) when the
//     element needs the accurate path, e.g. an FP32 result next to a zero of
//     the function, where its relative error would exceed the stated bound;
//   __device__ static void eval_rescue(int region, const T* in, T* out, uint32_t mask)
//     the accurate path.
// The declined elements of a tile are collected in shared memory and
// evaluated after the tile's groups, by consecutive threads, so that a few
// declined lanes do not hold a whole warp on the slow path.
template <class Fn, class = void>
struct HasRescue {
  static constexpr bool value = false;
};
template <class Fn>
struct HasRescue<Fn, decltype((void)Fn::RESCUE, void())> {
  static constexpr bool value = Fn::RESCUE;
};

// Evaluates the sorted tile in place.  Warps take the 32-slot groups of the
// sorted list dynamically from a shared counter, in list order: regions are
// numbered by decreasing cost, so the expensive groups start first and the
// tile's closing barrier waits on the cheapest ones.
template <class Fn, int TILE, bool AUX>
__device__ __forceinline__ void cta_eval_groups(int count, typename Fn::T* buf, const uint16_t* list,
                                                const uint8_t* regs, uint32_t mask, int* s_next, const double* aux0,
                                                int mode0, const double* aux1, int mode1) {
  using T = typename Fn::T;
  constexpr bool RESC = HasRescue<Fn>::value && !AUX;
  __shared__ uint16_t s_resc[RESC ? TILE : 1];
  __shared__ int s_nresc;
  const int lane = threadIdx.x & 31;
  const int ngroups = (count + 31) >> 5;
  if constexpr (RESC) {
    if (threadIdx.x == 0) s_nresc = 0;
    __syncthreads();
  }
  for (;;) {
    int gidx = 0;
    if (lane == 0) gidx = atomicAdd(s_next, 1);
    gidx = __shfl_sync(0xffffffffu, gidx, 0);
    if (gidx >= ngroups) break;
    const int j = (gidx << 5) + lane;
    bool declined = false;
    int li = 0;
    if (j < count) {
      li = list[j];
      T v[Fn::NIN], o[Fn::NOUT];
#pragma unroll
      for (int q = 0; q < Fn::NIN; ++q) v[q] = buf[q * TILE + li];
      bool done = true;
      if constexpr (AUX)
        Fn::eval(regs[li], v, o, mask, aux_at<Fn::NAUX0>(aux0, mode0, li), aux_at<Fn::NAUX1>(aux1, mode1, li));
      else if constexpr (RESC)
        done = Fn::eval_first(regs[li], v, o, mask);
      else
        Fn::eval(regs[li], v, o, mask);
      if (done) {
#pragma unroll
        for (int q = 0; q < Fn::NOUT; ++q) buf[q * TILE + li] = o[q];
      }
      declined = !done;
    }
    if constexpr (RESC) {
      // warp-aggregated push of the declined lanes' local indices
      const unsigned b = __ballot_sync(0xffffffffu, declined);
      if (b) {
        int base = 0;
        if (lane == __ffs(b) - 1) base = atomicAdd(&s_nresc, __popc(b));
        base = __shfl_sync(0xffffffffu, base, __ffs(b) - 1);
        if (declined) s_resc[base + __popc(b & ((1u << lane) - 1u))] = (uint16_t)li;
      }
    }
  }
  __syncthreads();
  if constexpr (RESC) {
    const int n = s_nresc;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const int li = s_resc[k];
      T v[Fn::NIN], o[Fn::NOUT];
#pragma unroll
      for (int q = 0; q < Fn::NIN; ++q) v[q] = buf[q * TILE + li];
      Fn::eval_rescue(regs[li], v, o, mask);
#pragma unroll
      for (int q = 0; q < Fn::NOUT; ++q) buf[q * TILE + li] = o[q];
    }
    __syncthreads();
  }
}

template <class Fn, typename TS>
__global__ void __launch_bounds__(kBlock, MinBlocks<Fn>::value) map_kernel(const MapParams<Fn::NIN, Fn::NOUT> p) {
  using T = typename Fn::T;
  using S = typename MapTile<Fn>::S;
  constexpr int NIN = Fn::NIN, NOUT = Fn::NOUT, R = Fn::R;
  constexpr int EPT = S::EPT, TILE = S::TILE;
  const int tid = threadIdx.x;
  const int64_t ntiles = (p.numel + TILE - 1) / TILE;

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
    __shared__ int s_cnt[R], s_base[R + 1], s_next;
    T* buf;
    uint16_t* list;
    uint8_t* regs;
    carve<S>(s_dyn, buf, list, regs);
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
          for (int q = 0; q < NIN; ++q) buf[q * TILE + li] = v[q];
        }
      }
      const int count = cta_sort_by_region<R, EPT>(reg, list, regs, s_cnt, s_base, &s_next);
      cta_eval_groups<Fn, TILE, false>(count, buf, list, regs, p.out_mask, &s_next, nullptr, 0, nullptr, 0);
#pragma unroll
      for (int k = 0; k < EPT; ++k) {
        const int li = k * kBlock + tid;
        const int64_t i = base + li;
        if (i < p.numel) {
          T o[NOUT];
#pragma unroll
          for (int q = 0; q < NOUT; ++q) o[q] = buf[q * TILE + li];
          store_element<Fn, TS>(p, i, o);
        }
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------ 2-D reduction
// 2-D tiles are 64 x 32 (2048 elements) when the staging fits in 64 KB,
// otherwise 32 x 32: more elements per tile spread each region's groups over
// more warps and amortise the tile's barriers and table fills.
// A functor with tables stages only its other inputs: the table inputs are
// read from their tables (or, when an input varies along both dimensions,
// again from global memory) at evaluation.
template <class Fn>
struct ReduceTile {
  static constexpr int NSTAGED = HasAux<Fn>::value ? Fn::NIN - 2 : Fn::NIN;
  // A single-region functor without tables is evaluated as its inputs are
  // loaded: only its outputs are staged (for the reductions and the stores).
  static constexpr bool EVAL_ON_LOAD = !HasAux<Fn>::value && Fn::R == 1;
  static constexpr int NBUF = EVAL_ON_LOAD ? Fn::NOUT : (NSTAGED > Fn::NOUT ? NSTAGED : Fn::NOUT);
  static constexpr int TR = TileRows<Fn>::value ? TileRows<Fn>::value
                                                : (Stage<Fn, 64 * kTC, NBUF>::SMEM <= 64 * 1024 ? 64 : kTRMin);
  static_assert(TR == 32 || TR == 64, "2-D tiles are 32 or 64 rows");
  using S = Stage<Fn, TR * kTC, NBUF>;
  // staging slot of input q (-1: a table input)
  __host__ __device__ static constexpr int slot(int q) {
    if (!HasAux<Fn>::value) return q;
    int k = 0;
    for (int i = 0; i < q; ++i)
      if (!is_table_input(i)) ++k;
    return is_table_input(q) ? -1 : k;
  }
  __host__ __device__ static constexpr bool is_table_input(int q) {
    if constexpr (HasAux<Fn>::value) return q == HasAuxIdx<Fn>::i0 || q == HasAuxIdx<Fn>::i1;
    return false;
  }
};
template <class Fn>
using ReduceStage = typename ReduceTile<Fn>::S;

template <class Fn, typename TS>
__global__ void __launch_bounds__(kBlock, MinBlocks<Fn>::value) reduce2d_kernel(const Reduce2DParams<Fn::NIN, Fn::NOUT> p) {
  using T = typename Fn::T;
  using S = ReduceStage<Fn>;
  constexpr int TR = ReduceTile<Fn>::TR;
  constexpr int NIN = Fn::NIN, NOUT = Fn::NOUT, R = Fn::R;
  constexpr int EPT = S::EPT, TILE = S::TILE;
  constexpr int RR = R > 1 ? R : 1;
  constexpr bool AUX = HasAux<Fn>::value;
  constexpr int N0 = HasAux<Fn>::N0, N1 = HasAux<Fn>::N1;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  __shared__ int s_cnt[RR], s_base[RR + 1], s_next;
  __shared__ double s_red[kBlock / 32][kTC];
  __shared__ double s_aux0[AUX ? TR * N0 : 1], s_aux1[AUX ? TR * N1 : 1];
  __shared__ T s_val0[AUX ? TR : 1], s_val1[AUX ? TR : 1];
  using RT = ReduceTile<Fn>;
  T* buf;
  uint16_t* list;
  uint8_t* regs;
  carve<S>(s_dyn, buf, list, regs);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t ntiles = p.n_row_tiles * p.n_col_tiles;
  int mode0 = 0, mode1 = 0;
  if constexpr (AUX) {
    mode0 = aux_mode(p.in_s0[Fn::AUX_IN0], p.in_s1[Fn::AUX_IN0]);
    mode1 = aux_mode(p.in_s0[Fn::AUX_IN1], p.in_s1[Fn::AUX_IN1]);
  }

  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t rt = t / p.n_col_tiles, ct = t % p.n_col_tiles;
    const int64_t r0 = rt * TR, c0 = ct * kTC;
    if constexpr (AUX) {
      // Tables for this tile: entries [0, TR) are input AUX_IN0's, [TR, 2TR)
      // input AUX_IN1's; a row table has TR entries, a column table kTC.
      for (int e = tid; e < 2 * TR; e += kBlock) {
        const int which = e / TR, j = e % TR, mode = which == 0 ? mode0 : mode1;
        if (mode == 0 || (mode == 2 && j >= kTC)) continue;
        const int64_t r = mode == 1 ? r0 + j : r0, c = mode == 1 ? c0 : c0 + j;
        if (r < p.rows && c < p.cols) {
          const int q = which == 0 ? Fn::AUX_IN0 : Fn::AUX_IN1;
          const T v = load_as<TS, T>(p.in_ptr[q] + (r * p.in_s0[q] + c * p.in_s1[q]) * (int64_t)sizeof(TS));
          if (which == 0) {
            s_val0[j] = v;
            Fn::make_aux0(v, s_aux0 + j * N0);
          } else {
            s_val1[j] = v;
            Fn::make_aux1(v, s_aux1 + j * N1);
          }
        }
      }
      __syncthreads();
    }
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
        if constexpr (RT::EVAL_ON_LOAD) {
          T o[NOUT];
          Fn::eval(0, v, o, p.out_mask);
#pragma unroll
          for (int q = 0; q < NOUT; ++q) buf[q * TILE + li] = o[q];
        } else {
          if constexpr (AUX) reg[k] = Fn::classify(v, aux_at<N0>(s_aux0, mode0, li), aux_at<N1>(s_aux1, mode1, li));
          else if constexpr (R > 1) reg[k] = Fn::classify(v);
          else reg[k] = 0;
#pragma unroll
          for (int q = 0; q < NIN; ++q)
            if (RT::slot(q) >= 0) buf[RT::slot(q) * TILE + li] = v[q];
        }
      }
    }
    if constexpr (AUX) {
      // As cta_eval_groups, with the table inputs taken from their tables.
      const int count = cta_sort_by_region<R, EPT>(reg, list, regs, s_cnt, s_base, &s_next);
      const int ngroups = (count + 31) >> 5;
      for (;;) {
        int gidx = 0;
        if (lane == 0) gidx = atomicAdd(&s_next, 1);
        gidx = __shfl_sync(0xffffffffu, gidx, 0);
        if (gidx >= ngroups) break;
        const int j = (gidx << 5) + lane;
        if (j < count) {
          const int li = list[j];
          const int lr = li / kTC, lc = li % kTC;
          T v[NIN], o[NOUT];
#pragma unroll
          for (int q = 0; q < NIN; ++q)
            if (RT::slot(q) >= 0) v[q] = buf[RT::slot(q) * TILE + li];
#pragma unroll
          for (int which = 0; which < 2; ++which) {
            const int q = which == 0 ? Fn::AUX_IN0 : Fn::AUX_IN1, mode = which == 0 ? mode0 : mode1;
            const T* tab = which == 0 ? s_val0 : s_val1;
            v[q] = mode == 1 ? tab[lr]
                 : mode == 2 ? tab[lc]
                             : load_as<TS, T>(p.in_ptr[q] + ((r0 + lr) * p.in_s0[q] + (c0 + lc) * p.in_s1[q]) *
                                                                (int64_t)sizeof(TS));
          }
          Fn::eval(regs[li], v, o, p.out_mask, aux_at<N0>(s_aux0, mode0, li), aux_at<N1>(s_aux1, mode1, li));
#pragma unroll
          for (int q = 0; q < NOUT; ++q) buf[q * TILE + li] = o[q];
        }
      }
      __syncthreads();
    } else if constexpr (R > 1) {
      const int count = cta_sort_by_region<R, EPT>(reg, list, regs, s_cnt, s_base, &s_next);
      cta_eval_groups<Fn, TILE, false>(count, buf, list, regs, p.out_mask, &s_next, nullptr, 0, nullptr, 0);
    } else {
      __syncthreads();  // single region: evaluated on load
    }

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
                         buf[o * TILE + li]);
        }
      } else if (kind == kOutRow || kind == kOutAll) {
        // Row sums: warp w takes rows w, w+8, ...; lane = column; fixed
        // shuffle tree.
        double tile_sum = 0.0;
        for (int lr = warp; lr < TR; lr += kBlock / 32) {
          double v = (lr < rows_here && lane < cols_here) ? (double)buf[o * TILE + lr * kTC + lane] : 0.0;
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
        // Column sums: warp w sums rows w, w+8, ... per lane (= column), then
        // the warp partials are added in warp order.
        double v = 0.0;
        for (int lr = warp; lr < rows_here; lr += kBlock / 32) v += (double)buf[o * TILE + lr * kTC + lane];
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

// Adds the partials of one reduced output: output i is the sum over k of
// ws[k * part_stride + i].  A CTA takes 32 outputs; its 8 warps each add
// every 8th partial (lane = output, so each load instruction of a warp reads
// 32 consecutive doubles), and warp 0 adds the 8 group sums in warp order,
// so the result does not depend on scheduling.
constexpr int kFinGroups = kBlock / 32;
template <typename TS>
__global__ void __launch_bounds__(kBlock) finalize_kernel(const double* ws, int64_t n_out, int64_t n_parts,
                                                          int64_t part_stride, char* out, int64_t out_stride) {
  __shared__ double s[kFinGroups][32];
  const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int64_t i = (int64_t)blockIdx.x * 32 + lane;
  double v = 0.0;
  if (i < n_out) {
#pragma unroll 4
    for (int64_t k = g; k < n_parts; k += kFinGroups) v += ws[k * part_stride + i];
  }
  s[g][lane] = v;
  __syncthreads();
  if (g == 0 && i < n_out) {
    double t = s[0][lane];
#pragma unroll
    for (int w = 1; w < kFinGroups; ++w) t += s[w][lane];
    store_as<TS>(out + i * out_stride * (int64_t)sizeof(TS), t);
  }
}

void count_launches(int64_t n);

// Launches finalize_kernel over n_out outputs (and counts the launch).
template <typename TS>
inline void launch_finalize(const double* ws, int64_t n_out, int64_t n_parts, int64_t part_stride, char* out,
                            int64_t out_stride, cudaStream_t stream) {
  const unsigned g = (unsigned)((n_out + 31) / 32);
  finalize_kernel<TS><<<g, kBlock, 0, stream>>>(ws, n_out, n_parts, part_stride, out, out_stride);
  count_launches(1);
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
