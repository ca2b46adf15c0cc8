// step_f64.cu -- FP64 fused step instantiations.  Built with -fmad=false so every product
// and sum rounds separately, as in the reference's x86-64 FP64 arithmetic.
#include "step_fp64.cuh"
#include "step_tma.cuh"
#include "step_batch.cuh"
#include "surface.cuh"

namespace mrlbm {

__global__ void __launch_bounds__(96) finish_record_kernel(const double* __restrict__ part, int nb, int ny, int halo_l,
                                                           double* rec, int iter) {
    __shared__ __align__(16) unsigned char smem[3 * AUX_CHUNK * sizeof(double)];
    record_sums(part, nb, ny, halo_l, rec, iter, smem);
}

int launch_finish_record(const double* partials, int nb, int ny, int halo_l, double* rec, int iter, void* stream) {
    finish_record_kernel<<<1, 96, 0, (cudaStream_t)stream>>>(partials, nb, ny, halo_l, rec, iter);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int launch_face_f64(const StepParams<double>& p, bool full, void* stream) {
    return full ? launch_face<fp64::Physics>(p, (cudaStream_t)stream)
                : launch_face<fp64::PhysicsLean>(p, (cudaStream_t)stream);
}

template <class Ph>
static int launch_step_impl(const StepParams<double>& p, int tile_cfg, cudaStream_t s, int workers) {
    switch (tile_cfg) {
#define MRLBM_TILE_CASE(id, bx, by, nj, mb64, mb32) \
    case id: return launch_step_tiles<Ph, bx, by, nj, mb64>(p, s);
        MRLBM_TILE_LIST(MRLBM_TILE_CASE)
#undef MRLBM_TILE_CASE
#define MRLBM_TMA_CASE(id, bx, by, st) \
    case id: return launch_step_tma<Ph, bx, by, st, false>(p, s, workers);
        MRLBM_TMA_LIST(MRLBM_TMA_CASE)
#undef MRLBM_TMA_CASE
#define MRLBM_TMAS_CASE(id, bx, by, st) \
    case id: return launch_step_tma<Ph, bx, by, st, true>(p, s, workers);
        MRLBM_TMAS_LIST(MRLBM_TMAS_CASE)
#undef MRLBM_TMAS_CASE
#define MRLBM_VEC_CASE(id, w, nj, mb) \
    case id: return launch_step_vec<Ph, w, nj, mb>(p, s);
        MRLBM_VEC_LIST(MRLBM_VEC_CASE)
#undef MRLBM_VEC_CASE
#define MRLBM_PIPE_CASE(id, b, mb) \
    case id: return launch_step_pipe<Ph, b, mb>(p, s);
        MRLBM_PIPE_LIST(MRLBM_PIPE_CASE)
#undef MRLBM_PIPE_CASE
    default: return -1;
    }
}

// The lean instantiation when the step has no field statistics, macroscopic output or body force.
int launch_step_f64(const StepParams<double>& p, int tile_cfg, void* stream, int workers) {
    cudaStream_t s = (cudaStream_t)stream;
    return (p.fstat || p.macro || p.body) ? launch_step_impl<fp64::Physics>(p, tile_cfg, s, workers)
                                          : launch_step_impl<fp64::PhysicsLean>(p, tile_cfg, s, workers);
}

int tma_ctas_per_sm_f64(int tile_cfg) {
    int n = 0;
    switch (tile_cfg) {
#define MRLBM_TMA_OCC(id, bx, by, st) \
    case id: n = tma_occupancy(step_kernel_tma<fp64::Physics, bx, by, st, false>, bx, tma_smem_bytes<double, bx, by, st, false>()); break;
        MRLBM_TMA_LIST(MRLBM_TMA_OCC)
#undef MRLBM_TMA_OCC
#define MRLBM_TMAS_OCC(id, bx, by, st) \
    case id: n = tma_occupancy(step_kernel_tma<fp64::Physics, bx, by, st, true>, bx, tma_smem_bytes<double, bx, by, st, true>()); break;
        MRLBM_TMAS_LIST(MRLBM_TMAS_OCC)
#undef MRLBM_TMAS_OCC
    default: n = 0;
    }
    return n;
}

template <class Ph>
static int launch_batch_impl(const BatchArgs<double>& a, int tile_cfg, int grid, bool cooperative, cudaStream_t s) {
    switch (tile_cfg) {
#define MRLBM_VEC_CASE(id, w, nj, mb) \
    case id: return launch_step_batch<Ph, w, nj, mb>(a, grid, cooperative, s);
        MRLBM_VEC_LIST(MRLBM_VEC_CASE)
#undef MRLBM_VEC_CASE
    default: return -2;
    }
}

int launch_batch_f64(const BatchArgs<double>& a, int tile_cfg, int grid, bool cooperative, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    return a.full ? launch_batch_impl<fp64::Physics>(a, tile_cfg, grid, cooperative, s)
                  : launch_batch_impl<fp64::PhysicsLean>(a, tile_cfg, grid, cooperative, s);
}

int batch_blocks_per_sm_f64(int tile_cfg) {
    using Ph = fp64::Physics;
    switch (tile_cfg) {
#define MRLBM_VEC_CASE(id, w, nj, mb) \
    case id: return batch_blocks_per_sm<Ph, w, nj, mb>();
        MRLBM_VEC_LIST(MRLBM_VEC_CASE)
#undef MRLBM_VEC_CASE
    default: return 0;
    }
}

int launch_surface_f64(const StepParams<double>& p, const SurfaceTables& t, double* rec, double* prec, cudaStream_t s) {
    return surf::launch_surface(p, t, rec, prec, s);
}

int launch_surface_f32(const StepParams<float>& p, const SurfaceTables& t, double* rec, double* prec, cudaStream_t s) {
    return surf::launch_surface(p, t, rec, prec, s);
}


template <class Ph>
static int launch_batch_split_impl(const BatchArgs<double>& a, int tile_cfg, int n_aux, int grid, cudaStream_t s) {
    switch (tile_cfg) {
#define MRLBM_TILE_CASE(id, bx, by, nj, mb64, mb32) \
    case id: return launch_batch_split<Ph, true, bx, by, nj, BATCH_MINB64[id]>(a, n_aux, grid, s);
        MRLBM_TILE_LIST(MRLBM_TILE_CASE)
#undef MRLBM_TILE_CASE
#define MRLBM_VEC_CASE(id, w, nj, mb) \
    case id: return launch_batch_split<Ph, false, w, 1, nj, BATCH_VEC_MINB64[id - VEC_CFG0]>(a, n_aux, grid, s);
        MRLBM_VEC_LIST(MRLBM_VEC_CASE)
#undef MRLBM_VEC_CASE
    default: return -2;
    }
}

int launch_batch_split_f64(const BatchArgs<double>& a, int tile_cfg, int n_aux, int grid, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    return a.full ? launch_batch_split_impl<fp64::Physics>(a, tile_cfg, n_aux, grid, s)
                  : launch_batch_split_impl<fp64::PhysicsLean>(a, tile_cfg, n_aux, grid, s);
}

int batch_split_blocks_per_sm_f64(int tile_cfg) {
    using Ph = fp64::PhysicsLean;
    switch (tile_cfg) {
#define MRLBM_TILE_CASE(id, bx, by, nj, mb64, mb32) \
    case id: return batch_split_per_sm<Ph, true, bx, by, nj, BATCH_MINB64[id]>();
        MRLBM_TILE_LIST(MRLBM_TILE_CASE)
#undef MRLBM_TILE_CASE
#define MRLBM_VEC_CASE(id, w, nj, mb) \
    case id: return batch_split_per_sm<Ph, false, w, 1, nj, BATCH_VEC_MINB64[id - VEC_CFG0]>();
        MRLBM_VEC_LIST(MRLBM_VEC_CASE)
#undef MRLBM_VEC_CASE
    default: return 0;
    }
}

}  // namespace mrlbm
