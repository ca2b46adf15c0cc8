// step_common.cuh -- launch skeleton shared by the FP64 and FP32 fused steps: pull-stream
// gather, coalesced store, tile mapping, boundary blocks and the per-step force reduction.
// The arithmetic of a node lives in a "physics" policy (step_fp64.cuh, step_fp32.cuh) with
//   static void bulk_node(const P&, int i, int j);
//   static void boundary_node(const P&, int l, double& Fx, double& Fy);
//   static double inlet_rho(const P&, int j);   // post-closure density of node (1,j)
#pragma once
#include <cuda_runtime.h>
#include "step_params.h"

namespace mrlbm {

// f(i,j,:) of this step = fout of the previous step at the streaming sources
// (stream_source in lattice.h).  Interior nodes take the branch-free fast path.
template <class T>
__device__ __forceinline__ void gather(const StepParams<T>& p, int i, int j, T f[Q]) {
    const int nx = p.L.nx, ny = p.L.ny;
    const int pitch = p.L.pitch, plane = (int)p.L.plane;
    if (i > 1 && i < nx && j > 1 && j < ny) {
        const T* s = p.src + ((int)(j * pitch + i + p.L.off));
#pragma unroll
        for (int k = 0; k < Q; ++k) f[k] = __ldg(s + (k * plane - ey(k) * pitch - ex(k)));
    } else {
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            SrcSlot sl = stream_source(nx, ny, i, j, k, p.xper, p.yper, p.freeslip);
            f[k] = __ldg(p.src + p.L.at(sl.i, sl.j, sl.k));
        }
        for (int q = 0; q < p.n_ovr; ++q)
            if (p.ovr[q].i == i && p.ovr[q].j == j) f[p.ovr[q].k] = (T)p.ovr[q].v;
    }
}

template <class T>
__device__ __forceinline__ void store(const StepParams<T>& p, int i, int j, const T fo[Q]) {
    T* d = p.dst + ((int)(j * p.L.pitch + i + p.L.off));
    const int plane = (int)p.L.plane;
#pragma unroll
    for (int k = 0; k < Q; ++k) d[k * plane] = fo[k];
}

template <class T>
__device__ __forceinline__ void store_macro(const StepParams<T>& p, int i, int j, double rho, double ux, double uy,
                                            double mxx, double myy, double mxy) {
    const int64_t n = (int64_t)(i - 1) + (int64_t)p.L.nx * (j - 1);
    const int64_t N = (int64_t)p.L.nx * p.L.ny;
    p.macro[n] = rho;
    p.macro[N + n] = ux;
    p.macro[2 * N + n] = uy;
    p.macro[3 * N + n] = mxx;
    p.macro[4 * N + n] = myy;
    p.macro[5 * N + n] = mxy;
}

// Node class inside the cylinder box: CLS_FLUID, CLS_SOLID or a boundary-node index.
template <class T>
__device__ __forceinline__ int node_class(const StepParams<T>& p, int i, int j) {
    const unsigned bx = (unsigned)(i - p.box_x0), by = (unsigned)(j - p.box_y0);
    if (bx < (unsigned)p.box_w && by < (unsigned)p.box_h) return __ldg(p.boxmap + by * p.box_w + bx);
    return CLS_FLUID;
}

// Boundary blocks own BNODES curved-wall nodes each, BLANES lanes per node.  The block first
// stages its nodes' tables in shared memory with coalesced loads.  Lane c of a node then
// pulls stencil node c (reference point 2 for c < 4, point 3 otherwise), computes its
// velocity and rotated moments, and the bilinear interpolation is completed with shuffles
// in the reference's operation order: (1-xd)*v1 + xd*v2 per row, then (1-yd)*a0 + yd*a1
// (2d_mrlbm.f90:786-793, 869-876).  Lane 0 runs the closure, collision, store and force.
constexpr int BNODES = 32;        // at most (256-thread blocks); blockDim.x / BLANES in general
constexpr int BLANES = 8;
constexpr int G_STAGED = G_SCC;   // GeoFields 0 .. G_SCC-1 live in shared memory

template <class T>
struct BTab {
    const T* g;
    const int* i;
    int n;                            // nodes per block (row stride of the staged tables)
    __device__ __forceinline__ T gf(int field, int li) const { return g[field * n + li]; }
    __device__ __forceinline__ int gi(int field, int li) const { return i[field * n + li]; }
};

template <class Phys>
__device__ __forceinline__ void boundary_block(const typename Phys::P& p) {
    using T = typename Phys::T;
    __shared__ T sg[G_STAGED * BNODES];
    __shared__ int sgi[I_NFIELDS * BNODES];
    __shared__ double sm[3 * 32];
    const int nthr = blockDim.x, tid = threadIdx.x;
    const int bn = nthr / BLANES;
    const int l0 = blockIdx.x * bn;
    for (int idx = tid; idx < G_STAGED * bn; idx += nthr) {
        const int f = idx / bn, n = idx - f * bn;
        sg[idx] = (l0 + n < p.nb) ? p.bgeo[f * p.nb + l0 + n] : T(0);
    }
    for (int idx = tid; idx < I_NFIELDS * bn; idx += nthr) {
        const int f = idx / bn, n = idx - f * bn;
        sgi[idx] = (l0 + n < p.nb) ? p.bint[f * p.nb + l0 + n] : 0;
    }
    __syncthreads();
    const BTab<T> tb{sg, sgi, bn};
    const int li = tid / BLANES, lane = tid % BLANES;
    const int l = l0 + li;
    const bool active = l < p.nb;
    const bool interp = p.closure == CLOSURE_UNROTATED || p.vel_interp || p.mom_interp;
    T ux = T(0), uy = T(0), mx = T(0), my = T(0);
    const int r = lane >> 2, c = lane & 3;        // reference point 2 + r, corner c
    const T xd = active ? tb.gf(r == 0 ? G_XD2 : G_XD3, li) : T(0);
    const T yd = active ? tb.gf(r == 0 ? G_YD2 : G_YD3, li) : T(0);
    if (active && interp) {
        const int s = 4 * r + c;
        const T cc = p.bgeo[(G_SCC + s) * p.nb + l], ss = p.bgeo[(G_SSS + s) * p.nb + l];
        const T s2 = p.bgeo[(G_SS2 + s) * p.nb + l];
        Phys::stencil_node(p, tb.gi(I_SI + s, li), tb.gi(I_SJ + s, li), cc, ss, s2, ux, uy, mx, my);
        const T wx = (c & 1) ? xd : (T(1) - xd);
        ux = wx * ux; uy = wx * uy; mx = wx * mx; my = wx * my;
    }
    const unsigned full = 0xffffffffu;
    // row sums (corner pairs 0+1, 2+3)
    ux = ux + __shfl_down_sync(full, ux, 1, BLANES);
    uy = uy + __shfl_down_sync(full, uy, 1, BLANES);
    mx = mx + __shfl_down_sync(full, mx, 1, BLANES);
    my = my + __shfl_down_sync(full, my, 1, BLANES);
    // column combination (1-yd)*a0 + yd*a1 at corners 0 (ref 2, lane 0) and 4 (ref 3, lane 4)
    {
        const T ux1 = __shfl_down_sync(full, ux, 2, BLANES), uy1 = __shfl_down_sync(full, uy, 2, BLANES);
        const T mx1 = __shfl_down_sync(full, mx, 2, BLANES), my1 = __shfl_down_sync(full, my, 2, BLANES);
        ux = (T(1) - yd) * ux + yd * ux1;
        uy = (T(1) - yd) * uy + yd * uy1;
        mx = (T(1) - yd) * mx + yd * mx1;
        my = (T(1) - yd) * my + yd * my1;
    }
    const T ux3 = __shfl_down_sync(full, ux, 4, BLANES), uy3 = __shfl_down_sync(full, uy, 4, BLANES);
    const T mx3 = __shfl_down_sync(full, mx, 4, BLANES), my3 = __shfl_down_sync(full, my, 4, BLANES);
    double Fx = 0.0, Fy = 0.0;
    if (active && lane == 0) {
        Phys::boundary_close(p, tb, li, l, ux, uy, mx, my, ux3, uy3, mx3, my3, Fx, Fy);
        if (p.do_stats) { p.partials[l] = Fx; p.partials[p.nb + l] = Fy; }
    }
    if (!p.do_stats) return;
    // rho(1,j) after the closures, for the inlet running mean (2d_mrlbm.f90:359)
    for (int j = 1 + blockIdx.x * nthr + tid; j <= p.L.ny; j += p.nbblk * nthr)
        p.partials[2 * p.nb + j - 1] = Phys::inlet_rho(p, j);
    // The last block to arrive sums the per-node forces and the inlet column in index order,
    // as the reference's sum() does (2d_mrlbm.f90:359, 488-489): the result does not depend on
    // the launch shape and equals the reference's sums bit for bit.
    __shared__ unsigned ticket;
    __threadfence();
    __syncthreads();
    if (tid == 0) ticket = atomicAdd(p.counter, 1u);
    __syncthreads();
    if (ticket != (unsigned)(p.nbblk - 1)) return;
    __threadfence();
    const int w = tid >> 5;
    if ((tid & 31) == 0 && w < 3) {
        const int n = w < 2 ? p.nb : p.L.ny;
        const double* v = p.partials + (w == 0 ? 0 : (w == 1 ? p.nb : 2 * p.nb));
        double acc = 0.0;
        for (int q = 0; q < n; ++q) acc = acc + __ldcg(v + q);
        sm[w] = acc;
    }
    __syncthreads();
    if (tid == 0) {
        if (p.rec) { p.rec[0] = (double)p.iter; p.rec[1] = sm[0]; p.rec[2] = sm[1]; p.rec[3] = sm[2]; }
        *p.counter = 0u;
    }
}

// Interior populations (no wraps, no ghosts): the branch-free half of `gather`.
template <class T>
__device__ __forceinline__ void gather_interior(const StepParams<T>& p, int i, int j, T f[Q]) {
    const int pitch = p.L.pitch, plane = (int)p.L.plane;
    const T* s = p.src + ((int)(j * pitch + i + p.L.off));
#pragma unroll
    for (int k = 0; k < Q; ++k) f[k] = __ldg(s + (k * plane - ey(k) * pitch - ex(k)));
}

// One time step.  Blocks [0, nbblk) are boundary blocks; the rest are bulk tiles of
// BX x (BY*NJ) nodes, one thread per column and NJ rows.  A thread first issues the loads of
// all its interior rows, then finishes them (collide and store) one by one, so up to 9*NJ
// loads per thread are in flight; edge rows and columns take the out-of-line edge path.
template <class Phys, int BX, int BY, int NJ, int MINB>
__global__ void __launch_bounds__(BX * BY, MINB) step_kernel(const __grid_constant__ typename Phys::P p) {
    using T = typename Phys::T;
    if ((int)blockIdx.x < p.nbblk) {
        boundary_block<Phys>(p);
        return;
    }
    const int t = blockIdx.x - p.nbblk;
    const int tx = t % p.tiles_x, ty = t / p.tiles_x;
    const int lx = threadIdx.x % BX, ly = threadIdx.x / BX;
    const int i = 1 + tx * BX + lx;
    const int nx = p.L.nx, ny = p.L.ny;
    if (i > nx) return;
    T f[NJ][Q];
    int cls[NJ];
    unsigned interior = 0u;
#pragma unroll
    for (int r = 0; r < NJ; ++r) {
        const int j = 1 + ty * BY * NJ + r * BY + ly;
        cls[r] = CLS_FLUID;
        if (j <= ny) {
            cls[r] = node_class(p, i, j);
            if (cls[r] < 0 && i > 1 && i < nx && j > 1 && j < ny) {
                gather_interior(p, i, j, f[r]);
                interior |= 1u << r;
            }
        }
    }
#pragma unroll
    for (int r = 0; r < NJ; ++r) {
        const int j = 1 + ty * BY * NJ + r * BY + ly;
        if ((interior >> r) & 1u) Phys::finish(p, i, j, cls[r], f[r]);
        else if (j <= ny && cls[r] < 0) Phys::edge_bulk_node(p, i, j, cls[r]);
    }
}

template <class Phys, int BX, int BY, int NJ, int MINB>
int launch_step_tiles(typename Phys::P p, cudaStream_t s) {
    const int nthr = BX * BY;
    static_assert(BX * BY % BLANES == 0 && BX * BY / BLANES <= BNODES, "boundary block size");
    const int bn = nthr / BLANES;
    p.nbblk = p.nb > 0 ? (p.nb + bn - 1) / bn : 1;
    p.tiles_x = (p.L.nx + BX - 1) / BX;
    const int tiles_y = (p.L.ny + BY * NJ - 1) / (BY * NJ);
    const long long nblocks = (long long)p.nbblk + (long long)p.tiles_x * tiles_y;
    step_kernel<Phys, BX, BY, NJ, MINB><<<(unsigned)nblocks, nthr, 0, s>>>(p);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace mrlbm
