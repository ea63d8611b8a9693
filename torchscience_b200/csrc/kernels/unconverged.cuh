// Count of elements whose bounded loop stopped at its iteration cap (the
// value is then a truncated sum).  Every math header whose loops are capped
// includes this; tsb_unconverged_count (abi.cu) reads the counters.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tsb {

// Host side: adds a unit's reader of its not-converged counter to the list
// that tsb_unconverged_count sums (abi.cu).
bool register_unconverged_reader(int64_t (*reader)(bool reset));

namespace {
// Elements whose series, continued fraction or recurrence stopped at its
// iteration cap, so that the result is a truncated sum (the loops are
// bounded: nothing waits on convergence).  Each translation unit and device
// has its own counter; tsb_unconverged_count adds them up.
__device__ unsigned long long g_unconverged = 0;

__device__ __forceinline__ void note_unconverged() { atomicAdd(&g_unconverged, 1ull); }

int64_t read_unconverged(bool reset) {
  unsigned long long v = 0;
  if (cudaMemcpyFromSymbol(&v, g_unconverged, sizeof(v)) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  if (reset && v) {
    const unsigned long long zero = 0;
    if (cudaMemcpyToSymbol(g_unconverged, &zero, sizeof(zero)) != cudaSuccess) cudaGetLastError();
  }
  return (int64_t)v;
}
const bool g_unconverged_registered = register_unconverged_reader(&read_unconverged);
}  // namespace

}  // namespace tsb
