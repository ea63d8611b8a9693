// torch.ops.torchscience_b200.unconverged_count: the C ABI's count of
// elements whose bounded loops stopped at their iteration cap.
#include <c10/cuda/CUDAGuard.h>
#include <torch/library.h>

#include "pointwise.h"

namespace tsbh {

int64_t unconverged_count(int64_t device, bool reset) {
  c10::cuda::CUDAGuard guard(static_cast<c10::DeviceIndex>(device));
  const int64_t n = tsb_unconverged_count(reset ? 1 : 0);
  TORCH_CHECK(n >= 0, "torchscience_b200 unconverged_count: ", tsb_status_string(static_cast<int32_t>(n)), ": ",
              tsb_last_error());
  return n;
}

}  // namespace tsbh

TORCH_LIBRARY_FRAGMENT(torchscience_b200, m) {
  m.def("unconverged_count(int device, bool reset) -> int", &tsbh::unconverged_count);
}
