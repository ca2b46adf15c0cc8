// step_f32.cu -- FP32 deviation-form fused step instantiations (contraction allowed).
#include "step_fp32.cuh"

namespace mrlbm {

int launch_step_f32(const StepParams<float>& p, int tile_cfg, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    using Ph = fp32::Physics;
    switch (tile_cfg) {
    case 0: return launch_step_tiles<Ph, 32, 8, 1, 4>(p, s);
    case 1: return launch_step_tiles<Ph, 32, 8, 2, 4>(p, s);
    case 2: return launch_step_tiles<Ph, 32, 4, 4, 8>(p, s);
    case 3: return launch_step_tiles<Ph, 64, 4, 2, 4>(p, s);
    default: return -1;
    }
}

}  // namespace mrlbm
