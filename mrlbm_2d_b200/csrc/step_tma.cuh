// step_tma.cuh -- persistent bulk tiles fed by TMA.
//
// Same time step as step_kernel (step_common.cuh); only the way interior populations reach
// the threads differs.  Bulk CTAs are persistent: each claims tiles of BX x BY nodes from a
// 64-bit counter and keeps STAGES tiles in flight in shared memory.  For a tile, one thread
// issues nine 2-D tensor copies (cp.async.bulk.tensor), one per direction plane k: the box
// of BY rows starting at row j0 - e_ky of plane k and BX + 2M columns starting M columns
// left of the tile (M = 16 bytes / element, so the box's x coordinate obeys the 16-byte rule),
// which holds exactly the pull-stream sources of plane k for every node of the tile.  The
// copies complete on the stage's mbarrier (expect_tx); threads wait on it, read their nine
// populations from shared memory, collide and store straight to global memory.  Edge and
// curved-wall nodes belong to the step's auxiliary launch, as with step_kernel.
//
// Every mbarrier wait is bounded: after TMA_SPIN_LIMIT polls the CTA raises errflag bit 4,
// drains its outstanding copies (again bounded) and returns.
#pragma once
#include <cuda.h>
#include "step_common.cuh"

namespace mrlbm {

constexpr unsigned TMA_SPIN_LIMIT = 1u << 26;
constexpr int ERR_TMA_TIMEOUT = 4;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait; false after TMA_SPIN_LIMIT polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    for (unsigned it = 0; it < TMA_SPIN_LIMIT; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            smem_u32(dst)),
        "l"((unsigned long long)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Tensor store shared -> global (bulk group), its commit and waits.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, const void* src, int x, int y) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                     (unsigned long long)map),
                 "r"(smem_u32(src)), "r"(x), "r"(y)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

template <class T, int BX, int BY>
struct TmaGeom {
    static constexpr int M = 16 / (int)sizeof(T);           // columns of margin each side
    static constexpr int W = BX + 2 * M;                      // box width (elements)
    static constexpr int ROW_BYTES = W * (int)sizeof(T);
    static constexpr int PLANE_BYTES = ((BY * ROW_BYTES + 127) / 128) * 128;
    static constexpr int STAGE_BYTES = Q * PLANE_BYTES;
    static constexpr unsigned TX_BYTES = (unsigned)(Q * BY * ROW_BYTES);
    static constexpr int OUT_PLANE = ((BY * BX * (int)sizeof(T) + 127) / 128) * 128;
    static constexpr int OUT_BYTES = Q * OUT_PLANE;       // output tile of the TMA-store shapes
    static_assert(W <= 256 && BY <= 256, "tensor copy box limit");
    static_assert((BX * (int)sizeof(T)) % 16 == 0, "box start must stay 16-byte aligned");
};

// Producer side: claim the next tile and start its nine plane copies into stage s.
template <class Phys, int BX, int BY>
__device__ __forceinline__ void tma_issue(const typename Phys::P& p, char* stage, uint64_t* bar, int* tile_slot,
                                          int ntiles) {
    using T = typename Phys::T;
    using G = TmaGeom<T, BX, BY>;
    const unsigned long long got = atomicAdd(p.tile_ctr, 1ull) - p.tile_base;
    const int t = got < (unsigned long long)ntiles ? (int)got : -1;
    *tile_slot = t;
    if (t < 0) {
        mbar_expect_tx(bar, 0u);                              // completes the phase: no more tiles
        return;
    }
    mbar_expect_tx(bar, G::TX_BYTES);
    const int tx = t % p.tiles_x, ty = t / p.tiles_x;
    const int x0 = (1 + tx * BX) + p.L.off - G::M;           // element column of the box start
    const int j0 = 1 + ty * BY;
    const int rows = p.L.ny + 2;
#pragma unroll
    for (int k = 0; k < Q; ++k)
        tma_load_2d(stage + k * G::PLANE_BYTES, &p.tmap, bar, x0, k * rows + j0 - ey(k));
}

template <class Phys, int BX, int BY, int STAGES, bool STORE>
__device__ __forceinline__ void tma_bulk_worker(const typename Phys::P& p) {
    using T = typename Phys::T;
    using G = TmaGeom<T, BX, BY>;
    extern __shared__ __align__(128) char tma_smem_raw[];
    // tensor copies need 128-byte aligned destinations; the launch adds 128 bytes of slack
    char* tma_smem = (char*)(((uintptr_t)tma_smem_raw + 127) & ~(uintptr_t)127);
    __shared__ __align__(8) uint64_t bars[STAGES];
    __shared__ int tile_of[STAGES];
    const int tid = threadIdx.x;
    const int ntiles = p.tiles_x * ((p.L.ny + BY - 1) / BY);
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
        fence_proxy_async();
    }
    __syncthreads();
    if (tid == 0)
        for (int s = 0; s < STAGES; ++s) tma_issue<Phys, BX, BY>(p, tma_smem + s * G::STAGE_BYTES, &bars[s], &tile_of[s], ntiles);
    const int nx = p.L.nx, ny = p.L.ny;
    T* out = reinterpret_cast<T*>(tma_smem + STAGES * G::STAGE_BYTES);   // STORE shapes only
    for (int q = 0;; ++q) {
        const int s = q % STAGES;
        const unsigned parity = (unsigned)(q / STAGES) & 1u;
        const bool ok = mbar_wait(&bars[s], parity);
        if (!__syncthreads_and(ok)) {
            if (tid == 0) {
                atomicOr(p.errflag, ERR_TMA_TIMEOUT);
                // let the copies still in flight land before the CTA's shared memory goes away:
                // the loads of the other stages (bounded waits) and the tensor stores committed
                // for earlier tiles, which still read the output tile
                for (int r = 1; r < STAGES; ++r) (void)mbar_wait(&bars[(q + r) % STAGES], (unsigned)((q + r) / STAGES) & 1u);
                if (STORE) bulk_wait_all();
            }
            __syncthreads();
            return;
        }
        const int t = tile_of[s];
        if (t < 0) break;                                     // tiles exhausted (later stages too)
        const T* st = reinterpret_cast<const T*>(tma_smem + s * G::STAGE_BYTES);
        const int tx = t % p.tiles_x, ty = t / p.tiles_x;
        const int i = 1 + tx * BX + tid;
        // a tile with no edge, ghost or cylinder-box node goes back through tensor stores
        const int i0 = 1 + tx * BX, j0 = 1 + ty * BY;
        const bool plain = plain_tile(p, i0, i0 + BX - 1, j0, j0 + BY - 1);
        const bool full = STORE && plain;
        if (full) {
            if (tid == 0) bulk_wait_read_all();               // the previous tile's stores have read `out`
            __syncthreads();
        }
#pragma unroll
        for (int r = 0; r < BY; ++r) {
            const int j = j0 + r;
            if (i > nx || j > ny) continue;
            T f[Q];
            if (full) {
#pragma unroll
                for (int k = 0; k < Q; ++k)
                    f[k] = st[(k * G::PLANE_BYTES) / (int)sizeof(T) + r * G::W + tid + G::M - ex(k)];
                T fo[Q];
                Phys::compute(p, i, j, CLS_FLUID, f, fo);
#pragma unroll
                for (int k = 0; k < Q; ++k) out[(k * G::OUT_PLANE) / (int)sizeof(T) + r * BX + tid] = fo[k];
                continue;
            }
            int cls = CLS_FLUID;
            if (!plain) {
                cls = node_class(p, i, j);
                if (cls >= 0) continue;                       // curved-wall node
                if (!is_interior(p, i, j)) continue;        // edge blocks
            }
#pragma unroll
            for (int k = 0; k < Q; ++k)
                f[k] = st[(k * G::PLANE_BYTES) / (int)sizeof(T) + r * G::W + tid + G::M - ex(k)];
            Phys::finish(p, i, j, cls, f);
        }
        __syncthreads();                                      // stage s fully read (and `out` written)
        if (tid == 0) {
            fence_proxy_async();
            if (full) {
                const int rows = p.L.ny + 2;
#pragma unroll
                for (int k = 0; k < Q; ++k)
                    tma_store_2d(&p.tmap_st, reinterpret_cast<const char*>(out) + k * G::OUT_PLANE, i0 + p.L.off,
                                 k * rows + j0);
                bulk_commit();
            }
            tma_issue<Phys, BX, BY>(p, tma_smem + s * G::STAGE_BYTES, &bars[s], &tile_of[s], ntiles);
        }
    }
    if (STORE && tid == 0) bulk_wait_all();                  // stores complete before the CTA exits
    // Every stage's last phase has completed: either its copies landed or it was issued with
    // no tile.  Nothing is in flight when the loop ends.
}

template <class Phys, int BX, int BY, int STAGES, bool STORE>
__global__ void __launch_bounds__(BX, 1) step_kernel_tma(const __grid_constant__ typename Phys::P p) {
    bulk_begin();
    tma_bulk_worker<Phys, BX, BY, STAGES, STORE>(p);
    bulk_end(p);
}

template <class T, int BX, int BY, int STAGES, bool STORE>
constexpr int tma_smem_bytes() {
    return STAGES * TmaGeom<T, BX, BY>::STAGE_BYTES + (STORE ? TmaGeom<T, BX, BY>::OUT_BYTES : 0) + 128;
}

template <class Phys, int BX, int BY, int STAGES, bool STORE>
int launch_step_tma(typename Phys::P p, cudaStream_t s, int workers) {
    if (workers <= 0) return -2;
    using T = typename Phys::T;
    using G = TmaGeom<T, BX, BY>;
    const int nthr = BX;
    p.tiles_x = (p.L.nx + BX - 1) / BX;
    const int smem = tma_smem_bytes<T, BX, BY, STAGES, STORE>();
    if (smem > 200 * 1024) return -2;                        // shape too large for this precision
    static unsigned long long attr_set = 0;                  // one bit per device
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64 || !((attr_set >> dev) & 1ull)) {
        if (cudaFuncSetAttribute(step_kernel_tma<Phys, BX, BY, STAGES, STORE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem) != cudaSuccess)
            return -1;
        if (dev < 64) attr_set |= 1ull << dev;
    }
    if (launch_aux<Phys>(p, s) != 0) return -1;
    p.nbblk = p.neblk = 0;
    return launch_after_prior(step_kernel_tma<Phys, BX, BY, STAGES, STORE>, (unsigned)workers,
                              nthr, (size_t)smem, s, p) == cudaSuccess
               ? 0
               : -1;
}

// Resident CTAs per SM of a TMA kernel with `smem` dynamic bytes: 0 when the shape does not
// fit, -(CUDA error) when a query fails.
template <class K>
int tma_occupancy(K kernel, int threads, int smem) {
    if (smem > 200 * 1024) return 0;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return -(int)e;
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem);
    if (e != cudaSuccess) return -(int)e;
    return n;
}

int tma_ctas_per_sm_f64(int tile_cfg);
int tma_ctas_per_sm_f32(int tile_cfg);

// Claims one TMA step makes on the tile counter: every tile once, plus exactly STAGES
// failing claims per worker (one per stage slot when the tiles run out).
inline unsigned long long tma_claims(int nx, int ny, int bx, int by, int stages, int workers) {
    return (unsigned long long)(((nx + bx - 1) / bx) * ((ny + by - 1) / by)) +
           (unsigned long long)workers * (unsigned long long)stages;
}

}  // namespace mrlbm
