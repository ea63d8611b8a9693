// Row-sorted sweep over a 2-D broadcast grid, for functors with per-input
// tables (HasAux) that opt in with `static constexpr bool SWEEP = true`.
//
// Layout it serves: input AUX_IN0 is constant along columns (an (R, 1)
// operand, e.g. the shape parameter a) and input AUX_IN1 constant along rows
// (a (1, C) operand, e.g. x), or the transpose of that; the other inputs and
// the outputs may be full, row-reduced, column-reduced or fully reduced.
//
// The cost of an element of the incomplete-gamma family depends on where
// (a, x) lies (series or continued fraction, and how many terms): a warp
// whose lanes hold unrelated a values runs as long as its slowest lane.  So:
//   1. sweep_setup_kernel sorts the R values of AUX_IN0 (a stable rank sort,
//      O(R^2) comparisons spread over the device) into `perm`;
//   2. sweep2d_kernel gives each warp a task of 32 consecutive sorted rows x
//      kSweepCols columns.  A lane owns one row: it builds that row's table
//      once per task, then walks the task's columns one at a time, every lane
//      at the same column.  The 32 lanes of a warp therefore share x and hold
//      nearly equal a: they take the same region and nearly the same number
//      of terms, with no per-tile sort and no block barrier.
//   3. full outputs are staged kSweepStage columns at a time in shared memory
//      and stored row-contiguously (32-byte runs for double); row-reduced
//      outputs accumulate in a register per lane (one partial per row and
//      task), column-reduced outputs are summed over the warp's 32 rows by a
//      fixed shuffle tree (one partial per column and row block), and the
//      partials are added in a fixed order by finalize_kernel, so results are
//      deterministic;
//   4. warps take tasks from a counter in the workspace (zeroed by the rank
//      kernel), the most expensive-looking row blocks (largest AUX_IN0) first.
// sweep_setup_kernel also computes the row table (quantities of a alone, e.g.
// lnΓ, ψ, ln a) of every sorted row and the column table (quantities of x
// alone) of every column into the workspace, so that the sweep kernel holds
// only the evaluation code; a task copies its 32 rows' entries into shared
// memory and the lanes read the column entry they share from global memory.
#pragma once

#include "dispatch.cuh"
#include "sweep_decl.cuh"

namespace tsb {

template <int NIN, int NOUT>
struct Sweep2DParams {
  int64_t rows, cols;                 // rows: the sorted dimension (AUX_IN0 varies along it)
  int64_t n_row_blocks, n_chunks;     // tasks = n_row_blocks x n_chunks
  char* in_ptr[NIN];
  int64_t in_s0[NIN], in_s1[NIN];     // element strides along rows / columns
  char* out_ptr[NOUT];
  int64_t out_s0[NOUT], out_s1[NOUT];
  int32_t out_kind[NOUT];
  double* ws[NOUT];                   // partial sums of reduced outputs
  int32_t* perm;                      // perm[k] = row of the k-th smallest AUX_IN0
  double* tab_rows;                   // [NAUX0][rows]: table of the k-th sorted row at [j * rows + k]
  double* tab_cols;                   // [cols][NAUX1]
  int32_t* counter;                   // next task (one counter per pass)
  uint32_t* colmask;                  // per task: the columns holding elements of a split sweep's second pass
  uint32_t out_mask;
};

// Storage type -> a type load_as can read it as (for the sort key).
template <typename TS> struct KeyT { using T = float; };
template <> struct KeyT<double> { using T = double; };

// Monotone map of a float to an unsigned integer (NaNs after +inf).
__device__ __forceinline__ unsigned int sweep_key(float v) {
  const unsigned int b = __float_as_uint(v);
  return (b >> 31) ? ~b : (b | 0x80000000u);
}

// Set-up of a sweep.  Blocks [0, row_blocks) take 32 rows each, one per
// lane: the row's rank among the AUX_IN0 values,
//   rank(i) = #{j : key_j < key_i} + #{j < i : key_j == key_i}
// (a stable sort), with the comparisons split over the block's warps (warp w
// counts over the w-th eighth of the keys, which its lanes load 32 at a time
// and pass round by shuffles), perm[rank] = i, and the row's table at sorted
// position rank.  The remaining blocks take one column per thread and fill
// its table.  Also zeroes the task counters.
template <class Fn, typename TS>
__global__ void __launch_bounds__(kBlock) sweep_setup_kernel(const Sweep2DParams<Fn::NIN, Fn::NOUT> p) {
  using T = typename Fn::T;
  using KT = typename KeyT<TS>::T;
  constexpr int IA = Fn::AUX_IN0, IX = Fn::AUX_IN1, N0 = Fn::NAUX0, W = kBlock / 32;
  const int64_t row_blocks = (p.rows + 31) / 32;
  if ((int64_t)blockIdx.x >= row_blocks) {
    const int64_t c = ((int64_t)blockIdx.x - row_blocks) * kBlock + threadIdx.x;
    if (c < p.cols)
      Fn::make_aux1(load_as<TS, T>(p.in_ptr[IX] + c * p.in_s1[IX] * (int64_t)sizeof(TS)), p.tab_cols + c * Fn::NAUX1);
    return;
  }
  __shared__ int s_part[W][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const char* key_ptr = p.in_ptr[IA];
  const int64_t key_stride = p.in_s0[IA] * (int64_t)sizeof(TS), n = p.rows;
  const int64_t i = (int64_t)blockIdx.x * 32 + lane;
  const unsigned int ki = i < n ? sweep_key((float)load_as<TS, KT>(key_ptr + i * key_stride)) : 0u;
  const int64_t per = (n + W - 1) / W, lo = warp * per, hi = lo + per < n ? lo + per : n;
  int cnt = 0;
  for (int64_t base = lo; base < hi; base += 32) {
    const int64_t jl = base + lane;
    const unsigned int kl = jl < hi ? sweep_key((float)load_as<TS, KT>(key_ptr + jl * key_stride)) : 0xffffffffu;
    const int m = (int)(hi - base < 32 ? hi - base : 32);
    for (int t = 0; t < m; ++t) {
      const unsigned int kj = __shfl_sync(0xffffffffu, kl, t);
      cnt += (kj < ki) | ((kj == ki) & (base + t < i));
    }
  }
  s_part[warp][lane] = cnt;
  __syncthreads();
  if (warp == 0 && i < n) {
    int64_t rank = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) rank += s_part[w][lane];
    p.perm[rank] = (int32_t)i;
    double tab[N0];
    Fn::make_aux0(load_as<TS, T>(key_ptr + i * key_stride), tab);
#pragma unroll
    for (int j = 0; j < N0; ++j) p.tab_rows[(int64_t)j * n + rank] = tab[j];
  }
  if (i == 0) p.counter[0] = p.counter[1] = 0;
}

// Resident CTAs per SM the sweep's register allocation must allow: a
// functor's SWEEP_MIN_BLOCKS, else 3 (85 registers: the task loop's state on
// top of the evaluator's; 4 CTAs would force spills at 64).
template <class Fn, class = void>
struct SweepMinBlocks {
  static constexpr int value = 3;
};
template <class Fn>
struct SweepMinBlocks<Fn, decltype((void)Fn::SWEEP_MIN_BLOCKS, void())> {
  static constexpr int value = Fn::SWEEP_MIN_BLOCKS;
};

template <class Fn>
struct SweepSmem {
  using T = typename Fn::T;
  static constexpr int W = kBlock / 32;
  static constexpr int N0P = Fn::NAUX0 | 1;  // odd stride in doubles: one lane per bank pair
  static constexpr size_t TAB = (size_t)W * 32 * N0P * sizeof(double);
  static constexpr size_t OUT = (size_t)W * Fn::NOUT * kSweepStage * 33 * sizeof(T);
  static constexpr size_t ACC = (size_t)W * Fn::NOUT * 32 * sizeof(double);  // row / all partials per lane
  static constexpr size_t OWN = (size_t)W * kSweepStage * 32;                 // staged element belongs to this pass
  static constexpr size_t BYTES = TAB + ACC + OUT + OWN;
  static_assert(Fn::NAUX0 <= kSweepTabMax && Fn::NAUX1 <= kSweepTabMax, "sweep tables too wide");
};

// PASS 0: every element (functors without a split); 1 and 2: the two passes
// of a split functor.  The FP32 pass fits 64 registers (4 resident CTAs).
template <class Fn, typename TS, int PASS>
__global__ void __launch_bounds__(kBlock, PASS == 1 ? 4 : SweepMinBlocks<Fn>::value)
    sweep2d_kernel(const Sweep2DParams<Fn::NIN, Fn::NOUT> p) {
  using T = typename Fn::T;
  using SM = SweepSmem<Fn>;
  constexpr int NIN = Fn::NIN, NOUT = Fn::NOUT, N0 = Fn::NAUX0, N1 = Fn::NAUX1, N0P = SM::N0P;
  constexpr int IA = Fn::AUX_IN0, IX = Fn::AUX_IN1, S = kSweepStage;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* tab = reinterpret_cast<double*>(s_dyn) + ((size_t)warp * 32 + lane) * N0P;
  double* acc = reinterpret_cast<double*>(s_dyn + SM::TAB) + (size_t)warp * NOUT * 32 + lane;  // [o][lane]
  T* so = reinterpret_cast<T*>(s_dyn + SM::TAB + SM::ACC) + (size_t)warp * NOUT * S * 33;  // [o][col][row]
  unsigned char* own = s_dyn + SM::TAB + SM::ACC + SM::OUT + (size_t)warp * S * 32;     // [col][row]
  const int ntasks = (int)(p.n_row_blocks * p.n_chunks);

  for (;;) {
    int task = 0;
    if (lane == 0) task = atomicAdd(p.counter + (PASS == 2 ? 1 : 0), 1);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= ntasks) break;
    // rows <= kSweepMaxRows: row indices fit in 32 bits
    const int rb = (int)p.n_row_blocks - 1 - task / (int)p.n_chunks, cc = task % (int)p.n_chunks;
    const bool rv = rb * 32 + lane < p.rows;
    const int r = p.perm[rv ? rb * 32 + lane : (int)p.rows - 1];
    const T a = load_as<TS, T>(p.in_ptr[IA] + (int64_t)r * p.in_s0[IA] * (int64_t)sizeof(TS));
    {
      const int kk = rv ? rb * 32 + lane : (int)p.rows - 1;
#pragma unroll
      for (int j = 0; j < N0; ++j) tab[j] = p.tab_rows[(int64_t)j * p.rows + kk];
    }
    const int64_t c0 = (int64_t)cc * kSweepCols;
    const int ncols = (int)(p.cols - c0 < kSweepCols ? p.cols - c0 : kSweepCols);
#pragma unroll
    for (int q = 0; q < NOUT; ++q) acc[q * 32] = 0.0;
    // The first pass of a split sweep records which of the task's columns
    // hold second-pass elements; the second pass visits only those.
    uint32_t cmask = 0u;
    if constexpr (PASS == 2) cmask = p.colmask[task];

    for (int jj = 0; jj < ncols; ++jj) {
      const int64_t col = c0 + jj;
      const int sj = jj % S;
      if (PASS == 2 && !((cmask >> jj) & 1u)) {  // no second-pass element in this column (warp-uniform)
        own[sj * 32 + lane] = 0;
      } else {
        const T x = load_as<TS, T>(p.in_ptr[IX] + col * p.in_s1[IX] * (int64_t)sizeof(TS));
        const double* xt = p.tab_cols + col * N1;  // every lane reads the same entry
        // classify and fp64_pass read only the two table inputs; the others
        // (e.g. an upstream gradient) are loaded for the elements this pass owns
        T v[NIN], o[NOUT];
        v[IA] = a;
        v[IX] = x;
        const int reg = Fn::classify(v, tab, xt);
        bool mine = true;
        if constexpr (PASS != 0) {
          const bool second = Fn::fp64_pass(reg, v, p.out_mask, tab, xt);
          mine = PASS == 2 ? second : !second;
          if constexpr (PASS == 1) {
            if (__any_sync(0xffffffffu, second)) cmask |= 1u << jj;
          }
        }
        if (mine) {
#pragma unroll
          for (int q = 0; q < NIN; ++q)
            if (q != IA && q != IX)
              v[q] = load_as<TS, T>(p.in_ptr[q] + ((int64_t)r * p.in_s0[q] + col * p.in_s1[q]) * (int64_t)sizeof(TS));
          if constexpr (PASS == 0) Fn::eval(reg, v, o, p.out_mask, tab, xt);
          else Fn::template eval_pass<PASS>(reg, v, o, p.out_mask, tab, xt);
        }
        const bool take = mine && rv;
        const unsigned any = __ballot_sync(0xffffffffu, take);
        own[sj * 32 + lane] = take;
#pragma unroll
        for (int q = 0; q < NOUT; ++q) {
          if (!(p.out_mask & (1u << q))) continue;
          const int kind = p.out_kind[q];
          if (kind == kOutFull) {
            if (take) so[(q * S + sj) * 33 + lane] = o[q];
          } else if (kind == kOutRow || kind == kOutAll) {
            if (take) acc[q * 32] += (double)o[q];
          } else if (kind == kOutCol) {
            // the first pass writes every partial, the second adds its own
            if (PASS != 2 || any) {
              double s = take ? (double)o[q] : 0.0;
#pragma unroll
              for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
              if (lane == 0) {
                double* w = p.ws[q] + (int64_t)rb * p.cols + col;
                *w = PASS == 2 ? *w + s : s;
              }
            }
          }
        }
      }
      __syncwarp();  // staged values visible to the storing lanes
      if (sj == S - 1 || jj == ncols - 1) {
        // Store the staged block: pass ps covers rows 8ps .. 8ps+7, lane -> (row lane / 4, column lane % 4).
        const int64_t cbase = col - sj;
#pragma unroll
        for (int q = 0; q < NOUT; ++q) {
          if (!(p.out_mask & (1u << q)) || p.out_kind[q] != kOutFull) continue;
#pragma unroll
          for (int ps = 0; ps < 32 * S / 32; ++ps) {
            const int i = ps * (32 / S) + lane / S, cj = lane % S;
            const int ri = __shfl_sync(0xffffffffu, r, i);
            if (cj <= sj && own[cj * 32 + i])
              store_as<TS>(p.out_ptr[q] + ((int64_t)ri * p.out_s0[q] + (cbase + cj) * p.out_s1[q]) * (int64_t)sizeof(TS),
                           so[(q * S + cj) * 33 + i]);
          }
        }
        __syncwarp();
      }
    }
    if constexpr (PASS == 1) {
      if (lane == 0) p.colmask[task] = cmask;
    }
#pragma unroll
    for (int q = 0; q < NOUT; ++q) {
      if (!(p.out_mask & (1u << q))) continue;
      if (p.out_kind[q] == kOutRow) {
        if (rv) {
          double* w = p.ws[q] + (int64_t)cc * p.rows + r;
          *w = PASS == 2 ? *w + acc[q * 32] : acc[q * 32];
        }
      } else if (p.out_kind[q] == kOutAll) {
        double s = acc[q * 32];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) p.ws[q][task] = PASS == 2 ? p.ws[q][task] + s : s;
      }
    }
  }
}

// Runs Fn through the row-sorted sweep (declared in dispatch.cuh).  Returns TSB_ERR_WORKSPACE
// without launching when `ws` is too small for the partial sums and the
// sweep's scratch, so that the caller can fall back to the tile kernel.
template <class Fn, typename TS>
int32_t launch_sweep(const Canon& c, bool transpose, const tsb_tensor* out, uint32_t mask, const tsb_tensor* in,
                     void* ws, int64_t ws_bytes, cudaStream_t stream, int dev, const DeviceInfo* info) {
  constexpr int NIN = Fn::NIN, NOUT = Fn::NOUT;
  Sweep2DParams<NIN, NOUT> p;
  const int d0 = transpose ? 1 : 0, d1 = 1 - d0;
  p.rows = c.size[d0];
  p.cols = c.size[d1];
  p.n_row_blocks = (p.rows + 31) / 32;
  p.n_chunks = (p.cols + kSweepCols - 1) / kSweepCols;
  p.out_mask = mask;
  const int64_t ntasks = p.n_row_blocks * p.n_chunks;
  if (ntasks >= (int64_t(1) << 31)) return set_error(TSB_ERR_LAYOUT, "grid too large for the sweep");
  for (int k = 0; k < NIN; ++k) {
    p.in_ptr[k] = static_cast<char*>(in[k].data);
    p.in_s0[k] = c.stride[k][d0];
    p.in_s1[k] = c.stride[k][d1];
  }
  char* wp = static_cast<char*>(ws);
  int64_t used = 0;
  for (int o = 0; o < NOUT; ++o) {
    const int k = NIN + o;
    p.out_ptr[o] = static_cast<char*>(out[o].data);
    p.ws[o] = nullptr;
    p.out_kind[o] = kOutNone;
    p.out_s0[o] = p.out_s1[o] = 0;
    if (!(mask & (1u << o))) continue;
    const int64_t s0 = c.stride[k][d0], s1 = c.stride[k][d1];
    p.out_s0[o] = s0;
    p.out_s1[o] = s1;
    int kind;
    int64_t n = 0;
    if (s0 != 0 && s1 != 0) kind = kOutFull;
    else if (s0 != 0) kind = kOutRow, n = p.n_chunks * p.rows;
    else if (s1 != 0) kind = kOutCol, n = p.n_row_blocks * p.cols;
    else kind = kOutAll, n = ntasks;
    p.out_kind[o] = kind;
    if (n > 0) {
      p.ws[o] = reinterpret_cast<double*>(wp + used);
      used += align256(n * (int64_t)sizeof(double));
    }
  }
  if (!ws || ((uintptr_t)ws % 256) != 0 || used + sweep_scratch_bytes(p.rows, p.cols) > ws_bytes)
    return TSB_ERR_WORKSPACE;
  char* sp = wp + used;
  p.perm = reinterpret_cast<int32_t*>(sp);
  sp += align256(p.rows * 4);
  p.tab_rows = reinterpret_cast<double*>(sp);
  p.tab_cols = p.tab_rows + p.rows * Fn::NAUX0;
  sp += align256((p.rows + p.cols) * kSweepTabMax * 8);
  p.colmask = reinterpret_cast<uint32_t*>(sp);
  p.counter = reinterpret_cast<int32_t*>(wp + used + sweep_scratch_bytes(p.rows, p.cols) - 256);

  const unsigned sgrid = (unsigned)((p.rows + 31) / 32 + (p.cols + kBlock - 1) / kBlock);
  sweep_setup_kernel<Fn, TS><<<sgrid, kBlock, 0, stream>>>(p);
  count_launches(1);
  int32_t st = check_launch("sweep set-up kernel launch");
  if (st) return st;
  constexpr size_t smem = SweepSmem<Fn>::BYTES;
  // one warp per task at most; persistent CTAs take tasks from the counter
  const int64_t warp_blocks = (ntasks + kBlock / 32 - 1) / (kBlock / 32);
  if constexpr (SplitOptIn<Fn>::value) {
    const int occ1 = occupancy_for<SweepTag<Fn, TS, 1>>(sweep2d_kernel<Fn, TS, 1>, kBlock, smem, dev);
    const int occ2 = occupancy_for<SweepTag<Fn, TS, 2>>(sweep2d_kernel<Fn, TS, 2>, kBlock, smem, dev);
    sweep2d_kernel<Fn, TS, 1><<<(unsigned)std::min<int64_t>(warp_blocks, (int64_t)info->sm_count * occ1), kBlock,
                                smem, stream>>>(p);
    sweep2d_kernel<Fn, TS, 2><<<(unsigned)std::min<int64_t>(warp_blocks, (int64_t)info->sm_count * occ2), kBlock,
                                smem, stream>>>(p);
    count_launches(2);
  } else {
    const int occ = occupancy_for<SweepTag<Fn, TS, 0>>(sweep2d_kernel<Fn, TS, 0>, kBlock, smem, dev);
    sweep2d_kernel<Fn, TS, 0><<<(unsigned)std::min<int64_t>(warp_blocks, (int64_t)info->sm_count * occ), kBlock,
                                smem, stream>>>(p);
    count_launches(1);
  }
  st = check_launch("sweep kernel launch");
  if (st) return st;
  for (int o = 0; o < NOUT; ++o) {
    if (!(p.out_mask & (1u << o))) continue;
    const int kind = p.out_kind[o];
    if (kind == kOutRow) {
      launch_finalize<TS>(p.ws[o], p.rows, p.n_chunks, p.rows, p.out_ptr[o], p.out_s0[o], stream);
    } else if (kind == kOutCol) {
      launch_finalize<TS>(p.ws[o], p.cols, p.n_row_blocks, p.cols, p.out_ptr[o], p.out_s1[o], stream);
    } else if (kind == kOutAll) {
      finalize_all_kernel<TS><<<1, kBlock, 0, stream>>>(p.ws[o], ntasks, p.out_ptr[o]);
      count_launches(1);
    } else {
      continue;
    }
    st = check_launch("finalize kernel launch");
    if (st) return st;
  }
  return TSB_OK;
}

}  // namespace tsb
