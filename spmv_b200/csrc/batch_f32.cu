// Instantiations of the lockstep batched kernel with FP32 inner iterations
// (mixed precision: FP64 refinement).
#include "batch_kernel.cuh"

namespace spmvb {
namespace bat {

bool launch_f32(const void* args, bool d16, const LaunchCfg& c, int num_sms, cudaStream_t s,
                bool dry) {
  if (d16) return launch_ci(*static_cast<const Args<float, int16_t>*>(args), c, num_sms, s, dry);
  return launch_ci(*static_cast<const Args<float, int32_t>*>(args), c, num_sms, s, dry);
}

}  // namespace bat
}  // namespace spmvb
