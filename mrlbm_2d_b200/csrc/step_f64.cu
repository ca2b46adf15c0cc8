// step_f64.cu -- FP64 fused step instantiations.  Built with -fmad=false so every product
// and sum rounds separately, as in the reference's x86-64 FP64 arithmetic.
#include "step_fp64.cuh"

namespace mrlbm {

int launch_step_f64(const StepParams<double>& p, int tile_cfg, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    using Ph = fp64::Physics;
    switch (tile_cfg) {   // minimum resident blocks sized for a 64-register budget
    case 0: return launch_step_tiles<Ph, 32, 8, 1, 4>(p, s);
    case 1: return launch_step_tiles<Ph, 32, 8, 2, 4>(p, s);
    case 2: return launch_step_tiles<Ph, 32, 4, 4, 8>(p, s);
    case 3: return launch_step_tiles<Ph, 64, 4, 2, 4>(p, s);
    default: return -1;
    }
}

}  // namespace mrlbm
