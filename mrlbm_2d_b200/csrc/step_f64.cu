// step_f64.cu -- FP64 fused step instantiations.  Built with -fmad=false so every product
// and sum rounds separately, as in the reference's x86-64 FP64 arithmetic.
#include "step_fp64.cuh"

namespace mrlbm {

template <int BX, int BY, int NJ>
static int launch_tiles(StepParams<double> p, cudaStream_t s) {
    const int nthr = BX * BY;
    p.nbblk = p.nb > 0 ? (p.nb + nthr - 1) / nthr : 1;
    p.tiles_x = (p.L.nx + BX - 1) / BX;
    const int tiles_y = (p.L.ny + BY * NJ - 1) / (BY * NJ);
    const long long nblocks = (long long)p.nbblk + (long long)p.tiles_x * tiles_y;
    fp64::step_kernel<BX, BY, NJ><<<(unsigned)nblocks, nthr, 0, s>>>(p);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int launch_step_f64(const StepParams<double>& p, int tile_cfg, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    switch (tile_cfg) {
    case 0: return launch_tiles<32, 8, 1>(p, s);
    case 1: return launch_tiles<32, 8, 2>(p, s);
    case 2: return launch_tiles<32, 4, 4>(p, s);
    case 3: return launch_tiles<64, 4, 2>(p, s);
    default: return -1;
    }
}

}  // namespace mrlbm
