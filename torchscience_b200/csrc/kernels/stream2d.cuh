// Streaming 2-D reduction for single-region, table-free functors that opt in
// with `static constexpr bool STREAM2D = true` (the backward from kept
// derivatives: grad · derivative, summed to the shape of each input).
//
// Such a pass does a few flops per element and is bound by HBM: on the
// 4096 x 4096 grid it reads three 134 MB operands.  The tiled 2-D kernel
// (reduce2d_kernel) stages each 64 x 32 tile through shared memory and keeps
// too few loads in flight for that; this kernel instead
//   * gives each CTA a band of kS2Rows rows x kS2Cols columns, each warp
//     kS2Rows / 8 of the band's rows, each lane kS2Per columns of a row at a
//     stride of 32 (every load instruction of a warp reads 256 contiguous
//     bytes of double data), so a lane has kS2Per independent loads per
//     operand in flight;
//   * sums row-reduced outputs across the lanes of a warp (fixed shuffle
//     tree) into one partial per (row, column band), and column-reduced
//     outputs over the band's rows (per lane, then over the warps in warp
//     order through shared memory) into one partial per (row band, column);
//   * stores full outputs directly;
// and finalize_kernel adds the partials in band order, so results are
// deterministic.  Inputs must be contiguous along the inner dimension; other
// layouts run through reduce2d_kernel.
#pragma once

#include "dispatch.cuh"

namespace tsb {

constexpr int kS2Rows = 32;   // rows per CTA band (kBlock / 32 warps take kS2Rows / 8 rows each)
constexpr int kS2Per = 8;     // columns per lane
constexpr int kS2Cols = 32 * kS2Per;

template <int NIN, int NOUT>
struct Stream2DParams {
  int64_t rows, cols, n_row_bands, n_col_bands;
  const char* in_ptr[NIN];
  int64_t in_s0[NIN];            // row strides (elements); the column stride is 1
  char* out_ptr[NOUT];
  int64_t out_s0[NOUT], out_s1[NOUT];
  int32_t out_kind[NOUT];
  double* ws[NOUT];              // kOutRow: [col band][row]; kOutCol: [row band][col]
};

template <class Fn, typename TS>
__global__ void __launch_bounds__(kBlock) stream2d_kernel(const Stream2DParams<Fn::NIN, Fn::NOUT> p) {
  using T = typename Fn::T;
  constexpr int NIN = Fn::NIN, NOUT = Fn::NOUT, W = kBlock / 32, RPW = kS2Rows / W;
  __shared__ double s_col[W][kS2Cols];  // per-warp column partials of one kOutCol output at a time
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t rb = blockIdx.x / p.n_col_bands, cb = blockIdx.x % p.n_col_bands;
  const int64_t c0 = cb * kS2Cols;
  double colacc[NOUT][kS2Per];
#pragma unroll
  for (int q = 0; q < NOUT; ++q)
#pragma unroll
    for (int j = 0; j < kS2Per; ++j) colacc[q][j] = 0.0;

  for (int i = 0; i < RPW; ++i) {
    const int64_t r = rb * kS2Rows + warp * RPW + i;
    if (r >= p.rows) break;  // warp-uniform
    T v[kS2Per][NIN];
#pragma unroll
    for (int j = 0; j < kS2Per; ++j) {
      const int64_t c = c0 + lane + 32 * j;
#pragma unroll
      for (int q = 0; q < NIN; ++q)
        v[j][q] = c < p.cols ? load_as<TS, T>(p.in_ptr[q] + (r * p.in_s0[q] + c) * (int64_t)sizeof(TS)) : T(0);
    }
    double rowacc[NOUT];
#pragma unroll
    for (int q = 0; q < NOUT; ++q) rowacc[q] = 0.0;
#pragma unroll
    for (int j = 0; j < kS2Per; ++j) {
      const int64_t c = c0 + lane + 32 * j;
      if (c >= p.cols) continue;
      T o[NOUT];
      Fn::eval(0, v[j], o, 0xffffffffu);
#pragma unroll
      for (int q = 0; q < NOUT; ++q) {
        const int kind = p.out_kind[q];
        if (kind == kOutRow) rowacc[q] += (double)o[q];
        else if (kind == kOutCol) colacc[q][j] += (double)o[q];
        else if (kind == kOutFull)
          store_as<TS>(p.out_ptr[q] + (r * p.out_s0[q] + c * p.out_s1[q]) * (int64_t)sizeof(TS), o[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < NOUT; ++q) {
      if (p.out_kind[q] != kOutRow) continue;
      double s = rowacc[q];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
      if (lane == 0) p.ws[q][cb * p.rows + r] = s;
    }
  }
#pragma unroll
  for (int q = 0; q < NOUT; ++q) {
    if (p.out_kind[q] != kOutCol) continue;  // uniform over the CTA
#pragma unroll
    for (int j = 0; j < kS2Per; ++j) s_col[warp][lane + 32 * j] = colacc[q][j];
    __syncthreads();
    for (int k = threadIdx.x; k < kS2Cols; k += kBlock) {
      const int64_t c = c0 + k;
      if (c >= p.cols) break;
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < W; ++w) s += s_col[w][k];
      p.ws[q][rb * p.cols + c] = s;
    }
    __syncthreads();
  }
}

// Workspace of the streaming reduction, or -1 when the layout does not suit it
// (inputs not contiguous along the inner dimension, or an output reduced
// along both dimensions).
inline int64_t stream2d_ws_bytes(const Canon& c, int n_in, const tsb_tensor* out, int n_out, uint32_t mask) {
  if (c.ndim != 2) return -1;
  for (int k = 0; k < n_in; ++k)
    if (c.stride[k][1] != 1) return -1;
  const int64_t nrb = (c.size[0] + kS2Rows - 1) / kS2Rows, ncb = (c.size[1] + kS2Cols - 1) / kS2Cols;
  int64_t need = 0;
  for (int o = 0; o < n_out; ++o) {
    if (!(mask & (1u << o))) continue;
    const int64_t s0 = c.stride[n_in + o][0], s1 = c.stride[n_in + o][1];
    if (s0 == 0 && s1 == 0) return -1;
    if (s1 == 0) need += align256(ncb * c.size[0] * (int64_t)sizeof(double));
    else if (s0 == 0) need += align256(nrb * c.size[1] * (int64_t)sizeof(double));
  }
  return need;
}

// Declared in dispatch.cuh.  Returns TSB_ERR_LAYOUT without launching when
// the layout or the workspace does not suit the streaming kernel.
template <class Fn, typename TS>
int32_t launch_stream2d(const Canon& c, const tsb_tensor* in, const tsb_tensor* out, uint32_t mask, void* ws,
                        int64_t ws_bytes, cudaStream_t stream) {
  constexpr int NIN = Fn::NIN, NOUT = Fn::NOUT;
  // Double storage only: on float data this layout measured slower than the
  // tiled kernel (1.1 TB/s against 1.4 on the 4096 x 4096 grid).
  if (sizeof(TS) != 8) return TSB_ERR_LAYOUT;
  const int64_t need = stream2d_ws_bytes(c, NIN, out, NOUT, mask);
  if (need < 0 || (need > 0 && (!ws || ws_bytes < need || ((uintptr_t)ws % 256) != 0))) return TSB_ERR_LAYOUT;
  Stream2DParams<NIN, NOUT> p;
  p.rows = c.size[0];
  p.cols = c.size[1];
  p.n_row_bands = (p.rows + kS2Rows - 1) / kS2Rows;
  p.n_col_bands = (p.cols + kS2Cols - 1) / kS2Cols;
  const int64_t blocks = p.n_row_bands * p.n_col_bands;
  if (blocks >= (int64_t(1) << 31)) return TSB_ERR_LAYOUT;
  for (int k = 0; k < NIN; ++k) {
    p.in_ptr[k] = static_cast<const char*>(in[k].data);
    p.in_s0[k] = c.stride[k][0];
  }
  char* wp = static_cast<char*>(ws);
  for (int o = 0; o < NOUT; ++o) {
    p.out_ptr[o] = static_cast<char*>(out[o].data);
    p.ws[o] = nullptr;
    p.out_kind[o] = kOutNone;
    p.out_s0[o] = p.out_s1[o] = 0;
    if (!(mask & (1u << o))) continue;
    const int64_t s0 = c.stride[NIN + o][0], s1 = c.stride[NIN + o][1];
    p.out_s0[o] = s0;
    p.out_s1[o] = s1;
    if (s0 != 0 && s1 != 0) {
      p.out_kind[o] = kOutFull;
    } else if (s1 == 0) {
      p.out_kind[o] = kOutRow;
      p.ws[o] = reinterpret_cast<double*>(wp);
      wp += align256(p.n_col_bands * p.rows * (int64_t)sizeof(double));
    } else {
      p.out_kind[o] = kOutCol;
      p.ws[o] = reinterpret_cast<double*>(wp);
      wp += align256(p.n_row_bands * p.cols * (int64_t)sizeof(double));
    }
  }
  stream2d_kernel<Fn, TS><<<(unsigned)blocks, kBlock, 0, stream>>>(p);
  count_launches(1);
  int32_t st = check_launch("streaming reduction kernel launch");
  if (st) return st;
  for (int o = 0; o < NOUT; ++o) {
    if (p.out_kind[o] == kOutRow) {
      launch_finalize<TS>(p.ws[o], p.rows, p.n_col_bands, p.rows, p.out_ptr[o], p.out_s0[o], stream);
    } else if (p.out_kind[o] == kOutCol) {
      launch_finalize<TS>(p.ws[o], p.cols, p.n_row_bands, p.cols, p.out_ptr[o], p.out_s1[o], stream);
    } else {
      continue;
    }
    st = check_launch("finalize kernel launch");
    if (st) return st;
  }
  return TSB_OK;
}

}  // namespace tsb
