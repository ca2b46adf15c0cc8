// step_batch.cuh -- many independent cylinder cases advanced by one kernel.
//
// Work items of one step, over all cases: first every case's boundary and edge blocks
// (aux items), then every case's bulk tiles of the 128-bit vector shape (step_common.cuh); a
// table gives the case of each item.
// A block copies the item's case parameters to shared memory, sets the per-step fields
// (time level, iteration, statistics flags, force-record slot) and runs the same device
// functions as the single-case kernels, so each case steps exactly as it would alone.
//
// Two schedules:
//   * persistent: one cooperative launch of resident blocks loops over the items of a step,
//     then meets the others at a grid barrier and goes on with the next step, for nsteps steps;
//   * per-step: one launch per step with one block per item (nsteps = 1), a sequence the
//     host captures in a CUDA graph and replays.
// Per-call state (iteration, time level, force-ring position) is uploaded before each call,
// so a captured graph replays correctly.  The grid barrier's wait is bounded: after
// BatchArgs::spin_limit polls (BAR_SPIN_LIMIT unless the host sets another limit) a block raises
// ERR_BARRIER_TIMEOUT, sets the abort flag that every waiting block also polls, and the kernel
// returns.
#pragma once
#include "batch_params.h"
#include <cstddef>
#include "step_common.cuh"

namespace mrlbm {

// Stats steps (post_process and statsbegin <= it <= statsend) among iterations a..b.
__device__ __forceinline__ int batch_stats_count(const BatchCase& c, int a, int b) {
    if (!c.post_process) return 0;
    const int lo = max(a, c.statsbegin), hi = min(b, c.statsend);
    return hi >= lo ? hi - lo + 1 : 0;
}

// Bounded grid barrier of a cooperative launch (all blocks resident).  False after an abort.
// A block that polls `limit` times without the generation moving raises ERR_BARRIER_TIMEOUT and
// the abort flag, which every other waiting block polls too, so the launch ends.
__device__ __forceinline__ bool batch_barrier(BatchBarrier* bar, unsigned limit) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = &bar->gen;
        volatile int* abort = &bar->abort;
        const unsigned g = *gen;
        __threadfence();
        ok = 1;
        if (atomicAdd(&bar->count, 1u) == gridDim.x - 1) {
            bar->count = 0u;
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            for (unsigned it = 0; *gen == g; ++it) {
                if (*abort) { ok = 0; break; }
                if (it >= limit) {
                    atomicOr(&bar->err, ERR_BARRIER_TIMEOUT);
                    atomicExch(&bar->abort, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

template <class Phys, int WARPS, int NJ, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) step_kernel_batch(const __grid_constant__ BatchArgs<typename Phys::T> a) {
    using T = typename Phys::T;
    using P = typename Phys::P;
    __shared__ __align__(64) unsigned char sp_raw[sizeof(P)];
    __shared__ __align__(16) unsigned char smem[aux_smem_bytes<T>()];
    P& sp = *reinterpret_cast<P*>(sp_raw);
    wait_prior_grid();                                   // per-step launches: see step_common.cuh
    const int n_aux = __ldg(a.aux_off + a.ncases);
    const int n_items = n_aux + __ldg(a.tile_off + a.ncases);
    for (int s = 0; s < a.nsteps; ++s) {
        const int cs = a.step0 + s;                     // step index within the call
        for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
            const bool aux = item < n_aux;
            const int c = __ldg(a.item_case + item);
            const int local = aux ? item - __ldg(a.aux_off + c) : item - n_aux - __ldg(a.tile_off + c);
            {   // case parameters -> shared memory, 16 bytes per thread
                const uint4* src = reinterpret_cast<const uint4*>(a.params + c);
                uint4* dst = reinterpret_cast<uint4*>(sp_raw);
                for (int q = threadIdx.x; q < (int)(sizeof(P) / 16); q += blockDim.x) dst[q] = src[q];
            }
            BatchCase bc;                                   // thread 0: loaded alongside the copy
            if (threadIdx.x == 0) bc = a.cases[c];
            __syncthreads();
            if (threadIdx.x == 0) {
                const int iter = bc.iter0 + cs + 1;
                if (cs & 1) {                           // params hold the call's first time level
                    const T* t = sp.src;
                    sp.src = sp.dst;
                    sp.dst = const_cast<T*>(t);
                }
                const bool stats = bc.post_process && iter >= bc.statsbegin && iter <= bc.statsend;
                sp.iter = iter;
                sp.do_stats = stats;
                sp.rec = stats ? bc.ring + (size_t)(bc.ring_n0 + batch_stats_count(bc, bc.iter0 + 1, iter - 1)) * REC_WORDS
                               : nullptr;
                sp.zero_solid_u = bc.post_process && bc.iplot > 0 && iter % bc.iplot == 0 && bc.plot_cyl;
                sp.macro = (a.want_macro && cs == a.call_steps - 1) ? bc.macro : nullptr;
                sp.fstat = (bc.fstat && iter >= bc.fs_begin && iter <= bc.fs_end) ? bc.fstat : nullptr;
                if (!(cs == 0 && bc.ovr_live)) {
                    sp.ovr = nullptr;
                    sp.n_ovr = 0;
                }
            }
            __syncthreads();
            if (aux) aux_item<Phys, wide_wall<Phys>(WARPS * 32, MINB)>(sp, smem, local);
            else vec_tile<Phys, WARPS, NJ>(sp, local);
            __syncthreads();
        }
        if (a.nsteps > 1 && !batch_barrier(a.bar, a.spin_limit)) return;
    }
}

// ---- split steps (graph schedule): an auxiliary launch and a bulk launch per step ----------
// The same ordering as a single case's step (step_common.cuh): the auxiliary launch waits for
// the previous step and lets the bulk launch start; the bulk launch's last block waits for the
// auxiliary launch.  A block stages the parameters of its case for this step in shared memory
// (the bytes after the tensor maps, which no batched path reads), with the per-step fields
// derived from the case's call state; a bulk block takes a contiguous run of tiles, so it
// stages again only when the run crosses into the next case.
template <class T>
__device__ __forceinline__ void batch_stage(const BatchArgs<T>& a, int c, int cs, unsigned char* sp_raw) {
    using P = StepParams<T>;
    constexpr int OFF = (int)offsetof(P, tile_ctr);
    static_assert(OFF % 16 == 0 && sizeof(P) % 16 == 0, "16-byte staging");
    P& sp = *reinterpret_cast<P*>(sp_raw);
    __syncthreads();                                   // the previous item is done with sp
    const uint4* src = reinterpret_cast<const uint4*>(reinterpret_cast<const char*>(a.params + c) + OFF);
    uint4* dst = reinterpret_cast<uint4*>(sp_raw + OFF);
    for (int q = threadIdx.x; q < (int)((sizeof(P) - OFF) / 16); q += blockDim.x) dst[q] = src[q];
    BatchCase bc;
    if (threadIdx.x == 0) bc = a.cases[c];
    __syncthreads();
    if (threadIdx.x == 0) {
        const int iter = bc.iter0 + cs + 1;
        if (cs & 1) {                                  // params hold the call's first time level
            const T* t = sp.src;
            sp.src = sp.dst;
            sp.dst = const_cast<T*>(t);
        }
        const bool stats = bc.post_process && iter >= bc.statsbegin && iter <= bc.statsend;
        sp.iter = iter;
        sp.do_stats = stats;
        sp.rec = stats ? bc.ring + (size_t)(bc.ring_n0 + batch_stats_count(bc, bc.iter0 + 1, iter - 1)) * REC_WORDS : nullptr;
        sp.zero_solid_u = bc.post_process && bc.iplot > 0 && iter % bc.iplot == 0 && bc.plot_cyl;
        sp.macro = (a.want_macro && cs == a.call_steps - 1) ? bc.macro : nullptr;
        sp.fstat = (bc.fstat && iter >= bc.fs_begin && iter <= bc.fs_end) ? bc.fstat : nullptr;
        if (!(cs == 0 && bc.ovr_live)) {
            sp.ovr = nullptr;
            sp.n_ovr = 0;
        }
    }
    __syncthreads();
}

static_assert(BATCH_AUX_THREADS == AUX_THREADS, "auxiliary block size of the split batch step");

template <class Phys>
__global__ void __launch_bounds__(AUX_THREADS) batch_aux_kernel(const __grid_constant__ BatchArgs<typename Phys::T> a) {
    using P = typename Phys::P;
    __shared__ __align__(64) unsigned char sp_raw[sizeof(P)];
    __shared__ __align__(16) unsigned char smem[aux_smem_bytes<typename Phys::T>()];
    wait_prior_grid();
    // a grid that fits the GPU at once walks all the cases' auxiliary items, so every block has
    // allowed the bulk launch to start within the first moments of the step
    const int n_aux = __ldg(a.aux_off + a.ncases);
    for (int item = (int)blockIdx.x; item < n_aux; item += (int)gridDim.x) {
        const int c = __ldg(a.aux_case + item);
        batch_stage(a, c, a.step0, sp_raw);
        aux_item<Phys, true, false>(*reinterpret_cast<const P*>(sp_raw), smem, item - __ldg(a.aux_off + c));
    }
}

// Bulk tiles of one split step.  TILE: a one-tile-per-block shape (BX x BY threads, NJ rows);
// otherwise a vector shape (BX warps, NJ rows per warp).
template <class Phys, bool TILE, int BX, int BY, int NJ, int MINB>
__global__ void __launch_bounds__(TILE ? BX * BY : BX * 32, MINB)
    batch_bulk_kernel(const __grid_constant__ BatchArgs<typename Phys::T> a) {
    using P = typename Phys::P;
    __shared__ __align__(64) unsigned char sp_raw[sizeof(P)];
    bulk_begin();
    const long long n = __ldg(a.tile_off + a.ncases);
    const int i0 = (int)(n * blockIdx.x / gridDim.x), i1 = (int)(n * (blockIdx.x + 1) / gridDim.x);
    if (i0 < i1) {
        // the case's tiles are consecutive items: a run needs the tile table only where it starts
        // and where it crosses into the next case (skipping cases without tiles)
        int c = __ldg(a.tile_case + i0);
        int t = i0 - __ldg(a.tile_off + c), end = __ldg(a.tile_off + c + 1);
        batch_stage(a, c, a.step0, sp_raw);
        const P& sp = *reinterpret_cast<const P*>(sp_raw);
        for (int item = i0; item < i1; ++item, ++t) {
            if (item == end) {
                do end = __ldg(a.tile_off + (++c) + 1);
                while (end == item);
                t = 0;
                batch_stage(a, c, a.step0, sp_raw);
            }
            if constexpr (TILE) tile_body<Phys, BX, BY, NJ>(sp, t);
            else vec_tile<Phys, BX, NJ>(sp, t);
        }
    }
    if (threadIdx.x == 0 && atomicAdd(&a.bar->bulk_done, 1u) == gridDim.x - 1) {
        a.bar->bulk_done = 0u;
        asm volatile("griddepcontrol.wait;" ::: "memory");
    }
}

template <class Phys, bool TILE, int BX, int BY, int NJ, int MINB>
int launch_batch_split(const BatchArgs<typename Phys::T>& a, int n_aux, int grid, cudaStream_t s) {
    if (launch_after_prior(batch_aux_kernel<Phys>, (unsigned)n_aux, AUX_THREADS, 0, s, a) != cudaSuccess) return -1;
    return launch_after_prior(batch_bulk_kernel<Phys, TILE, BX, BY, NJ, MINB>, (unsigned)grid, TILE ? BX * BY : BX * 32, 0, s,
                              a) == cudaSuccess
               ? 0
               : -1;
}

template <class Phys, bool TILE, int BX, int BY, int NJ, int MINB>
int batch_split_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_bulk_kernel<Phys, TILE, BX, BY, NJ, MINB>,
                                                      TILE ? BX * BY : BX * 32, 0) != cudaSuccess)
        return 0;
    return n;
}

// Block sizes and register budgets of the batch kernels: the vector shapes' (warps per block,
// resident blocks per SM).
template <class Phys, int WARPS, int NJ, int MINB>
int launch_step_batch(const BatchArgs<typename Phys::T>& a, int grid, bool cooperative, cudaStream_t s) {
    auto k = step_kernel_batch<Phys, WARPS, NJ, MINB>;
    if (!cooperative) return launch_after_prior(k, (unsigned)grid, WARPS * 32, 0, s, a) == cudaSuccess ? 0 : -1;
    void* args[] = {(void*)&a};
    return cudaLaunchCooperativeKernel((const void*)k, dim3((unsigned)grid), dim3(WARPS * 32), args, 0, s) ==
                   cudaSuccess
               ? 0
               : -1;
}

template <class Phys, int WARPS, int NJ, int MINB>
int batch_blocks_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, step_kernel_batch<Phys, WARPS, NJ, MINB>, WARPS * 32, 0) !=
        cudaSuccess)
        return 0;
    return n;
}

}  // namespace mrlbm
