// Library-wide C-ABI helpers: error state, device checks, workspace query.
#include <stdarg.h>
#include <stdio.h>

#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "dispatch.cuh"

namespace tsb {

namespace {
thread_local std::string g_last_error;
std::atomic<int64_t> g_launches{0};
std::mutex g_dev_mutex;
DeviceInfo g_devices[64];
bool g_dev_init[64];
}  // namespace

void count_launches(int64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {
std::mutex& unconverged_mutex() {
  static std::mutex m;
  return m;
}
std::vector<int64_t (*)(bool)>& unconverged_readers() {
  static std::vector<int64_t (*)(bool)> readers;
  return readers;
}
}  // namespace

bool register_unconverged_reader(int64_t (*reader)(bool reset)) {
  std::lock_guard<std::mutex> lock(unconverged_mutex());
  unconverged_readers().push_back(reader);
  return true;
}

int32_t set_error(int32_t status, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}

int32_t current_device(int* dev, const DeviceInfo** info) {
  int d = 0;
  cudaError_t e = cudaGetDevice(&d);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(TSB_ERR_DEVICE, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  }
  if (d < 0 || d >= 64) return set_error(TSB_ERR_DEVICE, "device ordinal %d out of range", d);
  {
    std::lock_guard<std::mutex> lock(g_dev_mutex);
    if (!g_dev_init[d]) {
      DeviceInfo di{};
      cudaDeviceGetAttribute(&di.sm_count, cudaDevAttrMultiProcessorCount, d);
      cudaDeviceGetAttribute(&di.major, cudaDevAttrComputeCapabilityMajor, d);
      cudaDeviceGetAttribute(&di.minor, cudaDevAttrComputeCapabilityMinor, d);
      e = cudaGetLastError();
      di.ok = e == cudaSuccess && di.major == 10 && di.minor == 0 && di.sm_count > 0;
      g_devices[d] = di;
      g_dev_init[d] = true;
    }
  }
  const DeviceInfo& di = g_devices[d];
  if (!di.ok)
    return set_error(TSB_ERR_DEVICE,
                     "device %d has compute capability %d.%d; these kernels are built for sm_100a (B200, 10.0) only", d,
                     di.major, di.minor);
  *dev = d;
  *info = &di;
  return TSB_OK;
}

}  // namespace tsb

extern "C" {

const char* tsb_version(void) { return "torchscience_b200 0.1.0 (sm_100a)"; }

int64_t tsb_launch_count(void) { return tsb::g_launches.load(std::memory_order_relaxed); }

int64_t tsb_unconverged_count(int32_t reset) {
  int dev = 0;
  const tsb::DeviceInfo* info = nullptr;
  const int32_t st = tsb::current_device(&dev, &info);
  if (st) return st;
  if (cudaDeviceSynchronize() != cudaSuccess) {
    const cudaError_t e = cudaGetLastError();
    return tsb::set_error(TSB_ERR_LAUNCH, "device synchronize failed: %s", cudaGetErrorString(e));
  }
  std::lock_guard<std::mutex> lock(tsb::unconverged_mutex());
  int64_t total = 0;
  for (auto* read : tsb::unconverged_readers()) {
    const int64_t v = read(reset != 0);
    if (v < 0) return tsb::set_error(TSB_ERR_DEVICE, "reading a not-converged counter failed");
    total += v;
  }
  return total;
}

const char* tsb_last_error(void) { return tsb::g_last_error.c_str(); }

const char* tsb_status_string(int32_t status) {
  switch (status) {
    case TSB_OK: return "ok";
    case TSB_ERR_ARGUMENT: return "invalid argument";
    case TSB_ERR_DTYPE: return "unsupported or mixed dtype";
    case TSB_ERR_LAYOUT: return "reduced-output layout not supported by the fused kernel";
    case TSB_ERR_WORKSPACE: return "workspace missing or too small";
    case TSB_ERR_LAUNCH: return "CUDA launch failure";
    case TSB_ERR_DEVICE: return "no usable sm_100 device";
    default: return "unknown status";
  }
}

int64_t tsb_workspace_bytes(const tsb_tensor* in, int32_t n_in, const tsb_tensor* out, int32_t n_out) {
  tsb::Canon c;
  int32_t dtype = 0;
  const int32_t st = tsb::canonicalize(in, n_in, out, n_out, n_in, n_out, c, dtype);
  if (st) return st;
  bool reduced = false;
  for (int o = 0; o < n_out; ++o)
    if (out[o].data && tsb::output_is_reduced(c, n_in + o)) reduced = true;
  // A 2-D grid with an input constant along each dimension ((R, 1) x (1, C)):
  // room for the row-sorted sweep's row order, row and column tables and
  // task counter, which the functions with per-input tables use when given.
  int64_t sweep = 0;
  if (c.numel > 0 && c.ndim == 2) {
    bool row_const = false, col_const = false;
    for (int k = 0; k < n_in; ++k) {
      row_const |= c.stride[k][0] != 0 && c.stride[k][1] == 0;
      col_const |= c.stride[k][0] == 0 && c.stride[k][1] != 0;
    }
    if (row_const && col_const) sweep = tsb::sweep_scratch_bytes(c.size[0], c.size[1]);
  }
  if (!reduced) return sweep;
  if (c.ndim > 2)
    return tsb::set_error(TSB_ERR_LAYOUT, "reduced outputs need an iteration space of at most 2 coalesced dims");
  return tsb::reduce_ws_bytes(c, n_in, out, n_out, tsb::kTRMin) + sweep;
}

}  // extern "C"
