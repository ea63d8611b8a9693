// Declarations of the row-sorted sweep (sweep.cuh) that every entry point's
// dispatch and the workspace query need: the functor opt-in traits, the
// sweep's size limits and its scratch size.  The kernels and their launcher
// are in sweep.cuh, which only the units of functors that opt in include.
#pragma once

#include <stdint.h>

namespace tsb {

template <class Fn, class = void>
struct SweepOptIn {
  static constexpr bool value = false;
};
template <class Fn>
struct SweepOptIn<Fn, decltype((void)Fn::SWEEP, void())> {
  static constexpr bool value = Fn::SWEEP;
};

// Functors that split a sweep into two passes: `SPLIT`, fp64_pass(region,
// in, mask, A, X) (whether an element belongs to the second pass) and
// eval_pass<1 or 2>(...).  The first pass runs compact FP32 code over the
// elements it can take and writes every reduced partial; the second runs the
// FP64 evaluator over the rest and adds to the partials (in that order, so
// results are deterministic).  Kept apart, each kernel's code fits the
// instruction cache, which a kernel holding both precisions' evaluators
// does not.
template <class Fn, class = void>
struct SplitOptIn {
  static constexpr bool value = false;
};
template <class Fn>
struct SplitOptIn<Fn, decltype((void)Fn::SPLIT, void())> {
  static constexpr bool value = Fn::SPLIT;
};

constexpr int kSweepCols = 32;             // columns per task
static_assert(kSweepCols == 32, "a task's column mask is one 32-bit word");
constexpr int kSweepStage = 4;             // full-output columns staged per store
constexpr int64_t kSweepMaxRows = 16384;   // the rank sort is O(rows^2): larger grids use reduce2d_kernel

// Per-row / per-column table entries the sweep keeps in its workspace (a
// functor's NAUX0, NAUX1 must not exceed this many doubles).
constexpr int kSweepTabMax = 16;

// Scratch the sweep needs beyond the reduced outputs' partial sums, for a grid
// of n0 x n1 (either orientation): the row order (int32 per sorted row), the
// row and column tables (kSweepTabMax doubles per row and per column), one
// 32-bit column mask per task (the columns a split sweep's second pass
// visits; tasks are 32 rows x kSweepCols = 32 columns) and the task counters.
inline int64_t sweep_task_count(int64_t n0, int64_t n1) { return ((n0 + 31) / 32) * ((n1 + 31) / 32); }
inline int64_t sweep_scratch_bytes(int64_t n0, int64_t n1) {
  const int64_t rows = n0 > n1 ? n0 : n1;
  return ((rows * 4 + 255) & ~int64_t(255)) + (((n0 + n1) * kSweepTabMax * 8 + 255) & ~int64_t(255)) +
         ((sweep_task_count(n0, n1) * 4 + 255) & ~int64_t(255)) + 256;
}

}  // namespace tsb
