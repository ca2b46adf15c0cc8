// step_f32.cu -- FP32 deviation-form fused step (populations stored as f_k - w_k).
#include <cuda_runtime.h>
#include "step_params.h"

namespace mrlbm {
int launch_step_f32(const StepParams<float>&, int, void*) { return -1; }
}  // namespace mrlbm
