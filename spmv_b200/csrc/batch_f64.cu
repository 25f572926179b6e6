// Instantiations of the lockstep batched kernel with FP64 inner iterations
// (plain FP64 CG with a confirming FP64 residual at the end).
#include "batch_kernel.cuh"

namespace spmvb {
namespace bat {

bool launch_f64(const void* args, bool d16, const LaunchCfg& c, int num_sms, cudaStream_t s,
                bool dry) {
  if (d16) return launch_ci(*static_cast<const Args<double, int16_t>*>(args), c, num_sms, s, dry);
  return launch_ci(*static_cast<const Args<double, int32_t>*>(args), c, num_sms, s, dry);
}

}  // namespace bat
}  // namespace spmvb
