// step_f32.cu -- FP32 deviation-form fused step instantiations (contraction allowed).
#include "step_fp32.cuh"
#include "step_tma.cuh"
#include "step_batch.cuh"

namespace mrlbm {

int launch_face_f32(const StepParams<float>& p, bool full, void* stream) {
    return full ? launch_face<fp32::Physics>(p, (cudaStream_t)stream)
                : launch_face<fp32::PhysicsLean>(p, (cudaStream_t)stream);
}

template <class Ph>
static int launch_step_impl(const StepParams<float>& p, int tile_cfg, cudaStream_t s, int workers) {
    switch (tile_cfg) {
#define MRLBM_TILE_CASE(id, bx, by, nj, mb64, mb32) \
    case id: return launch_step_tiles<Ph, bx, by, nj, mb32>(p, s);
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
int launch_step_f32(const StepParams<float>& p, int tile_cfg, void* stream, int workers) {
    cudaStream_t s = (cudaStream_t)stream;
    return (p.fstat || p.macro || p.body) ? launch_step_impl<fp32::Physics>(p, tile_cfg, s, workers)
                                          : launch_step_impl<fp32::PhysicsLean>(p, tile_cfg, s, workers);
}

int tma_ctas_per_sm_f32(int tile_cfg) {
    int n = 0;
    switch (tile_cfg) {
#define MRLBM_TMA_OCC(id, bx, by, st) \
    case id: n = tma_occupancy(step_kernel_tma<fp32::Physics, bx, by, st, false>, bx, tma_smem_bytes<float, bx, by, st, false>()); break;
        MRLBM_TMA_LIST(MRLBM_TMA_OCC)
#undef MRLBM_TMA_OCC
#define MRLBM_TMAS_OCC(id, bx, by, st) \
    case id: n = tma_occupancy(step_kernel_tma<fp32::Physics, bx, by, st, true>, bx, tma_smem_bytes<float, bx, by, st, true>()); break;
        MRLBM_TMAS_LIST(MRLBM_TMAS_OCC)
#undef MRLBM_TMAS_OCC
    default: n = 0;
    }
    return n;
}

int tma_ctas_per_sm(int precision, int tile_cfg) {
    return precision == 64 ? tma_ctas_per_sm_f64(tile_cfg) : tma_ctas_per_sm_f32(tile_cfg);
}

void tma_box(int precision, int tile_cfg, int* box_w, int* box_h, int* stages) {
    const TmaCfg c = tma_cfg(tile_cfg);
    const int m = 16 / (precision == 64 ? 8 : 4);
    *box_w = c.bx + 2 * m;
    *box_h = c.by;
    *stages = c.stages;
}

template <class Ph>
static int launch_batch_impl(const BatchArgs<float>& a, int tile_cfg, int grid, bool cooperative, cudaStream_t s) {
    switch (tile_cfg) {
#define MRLBM_VEC_CASE(id, w, nj, mb) \
    case id: return launch_step_batch<Ph, w, nj, mb>(a, grid, cooperative, s);
        MRLBM_VEC_LIST(MRLBM_VEC_CASE)
#undef MRLBM_VEC_CASE
    default: return -2;
    }
}

int launch_batch_f32(const BatchArgs<float>& a, int tile_cfg, int grid, bool cooperative, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    return a.full ? launch_batch_impl<fp32::Physics>(a, tile_cfg, grid, cooperative, s)
                  : launch_batch_impl<fp32::PhysicsLean>(a, tile_cfg, grid, cooperative, s);
}

int batch_blocks_per_sm_f32(int tile_cfg) {
    using Ph = fp32::Physics;
    switch (tile_cfg) {
#define MRLBM_VEC_CASE(id, w, nj, mb) \
    case id: return batch_blocks_per_sm<Ph, w, nj, mb>();
        MRLBM_VEC_LIST(MRLBM_VEC_CASE)
#undef MRLBM_VEC_CASE
    default: return 0;
    }
}

int batch_blocks_per_sm(int precision, int tile_cfg) {
    return precision == 64 ? batch_blocks_per_sm_f64(tile_cfg) : batch_blocks_per_sm_f32(tile_cfg);
}

int batch_split_blocks_per_sm(int precision, int tile_cfg) {
    return precision == 64 ? batch_split_blocks_per_sm_f64(tile_cfg) : batch_split_blocks_per_sm_f32(tile_cfg);
}

int batch_split_threads(int tile_cfg) {
    switch (tile_cfg) {
#define MRLBM_TILE_CASE(id, bx, by, nj, mb64, mb32) \
    case id: return bx * by;
        MRLBM_TILE_LIST(MRLBM_TILE_CASE)
#undef MRLBM_TILE_CASE
#define MRLBM_VEC_CASE(id, w, nj, mb) \
    case id: return w * 32;
        MRLBM_VEC_LIST(MRLBM_VEC_CASE)
#undef MRLBM_VEC_CASE
    default: return 0;
    }
}

int batch_block_threads(int tile_cfg) {
    switch (tile_cfg) {
#define MRLBM_VEC_CASE(id, w, nj, mb) \
    case id: return w * 32;
        MRLBM_VEC_LIST(MRLBM_VEC_CASE)
#undef MRLBM_VEC_CASE
    default: return 0;
    }
}


template <class Ph>
static int launch_batch_split_impl(const BatchArgs<float>& a, int tile_cfg, int n_aux, int grid, cudaStream_t s) {
    switch (tile_cfg) {
#define MRLBM_TILE_CASE(id, bx, by, nj, mb64, mb32) \
    case id: return launch_batch_split<Ph, true, bx, by, nj, BATCH_MINB32[id]>(a, n_aux, grid, s);
        MRLBM_TILE_LIST(MRLBM_TILE_CASE)
#undef MRLBM_TILE_CASE
#define MRLBM_VEC_CASE(id, w, nj, mb) \
    case id: return launch_batch_split<Ph, false, w, 1, nj, BATCH_VEC_MINB32[id - VEC_CFG0]>(a, n_aux, grid, s);
        MRLBM_VEC_LIST(MRLBM_VEC_CASE)
#undef MRLBM_VEC_CASE
    default: return -2;
    }
}

int launch_batch_split_f32(const BatchArgs<float>& a, int tile_cfg, int n_aux, int grid, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    return a.full ? launch_batch_split_impl<fp32::Physics>(a, tile_cfg, n_aux, grid, s)
                  : launch_batch_split_impl<fp32::PhysicsLean>(a, tile_cfg, n_aux, grid, s);
}

int batch_split_blocks_per_sm_f32(int tile_cfg) {
    using Ph = fp32::PhysicsLean;
    switch (tile_cfg) {
#define MRLBM_TILE_CASE(id, bx, by, nj, mb64, mb32) \
    case id: return batch_split_per_sm<Ph, true, bx, by, nj, BATCH_MINB32[id]>();
        MRLBM_TILE_LIST(MRLBM_TILE_CASE)
#undef MRLBM_TILE_CASE
#define MRLBM_VEC_CASE(id, w, nj, mb) \
    case id: return batch_split_per_sm<Ph, false, w, 1, nj, BATCH_VEC_MINB32[id - VEC_CFG0]>();
        MRLBM_VEC_LIST(MRLBM_VEC_CASE)
#undef MRLBM_VEC_CASE
    default: return 0;
    }
}

}  // namespace mrlbm
