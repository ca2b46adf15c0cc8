// step_common.cuh -- launch skeleton shared by the FP64 and FP32 fused steps: pull-stream
// gather, coalesced store, tile mapping, boundary and edge blocks and the per-step force
// reduction.  The arithmetic of a node lives in a "physics" policy (step_fp64.cuh,
// step_fp32.cuh) with
//   static void compute(const P&, int i, int j, int cls, const T f[Q], T fo[Q]);  // bulk node
//   static void finish(const P&, int i, int j, int cls, const T f[Q]);            // compute + store
//   static double edge_bulk_node(const P&, int i, int j, int cls);  // edge node; returns rho
//   static void stencil_node(...), boundary_close(...);               // curved-wall nodes
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include "step_params.h"

namespace mrlbm {

// Programmatic dependent launch.  The step kernels are launched with programmatic stream
// serialization.  Each block first waits for the previous kernel on the stream to complete
// and its writes to be visible (griddepcontrol.wait; at once when there is none), then allows
// the next kernel to launch (griddepcontrol.launch_dependents): once every block of this grid
// is running, the next step's blocks are dispatched onto the SM slots this grid frees and
// wait there, so its launch overlaps this step's tail.  Nothing a step reads or writes is
// touched before the wait.
__device__ __forceinline__ void wait_prior_grid() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <class K, class... A>
inline cudaError_t launch_after_prior(K kernel, unsigned grid, unsigned block, size_t smem, cudaStream_t s, const A&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Columns 1 and nx are domain edges unless the lattice is one x-slab of a larger domain and
// the neighbouring slab supplies that side's incoming populations in column 0 / nx+1.
template <class T>
__device__ __forceinline__ bool col_interior(const StepParams<T>& p, int i) {
    return (i > 1 || p.halo_l) && (i < p.L.nx || p.halo_r);
}
template <class T>
__device__ __forceinline__ bool is_interior(const StepParams<T>& p, int i, int j) {
    return col_interior(p, i) && j > 1 && j < p.L.ny;
}

// f(i,j,:) of this step = fout of the previous step at the streaming sources
// (stream_source in lattice.h).  Interior nodes take the branch-free fast path.
template <class T>
__device__ __forceinline__ void gather(const StepParams<T>& p, int i, int j, T f[Q]) {
    const int nx = p.L.nx, ny = p.L.ny;
    const int pitch = p.L.pitch, plane = (int)p.L.plane;
    if (is_interior(p, i, j)) {
        const T* s = p.src + ((int)(j * pitch + i + p.L.off));
#pragma unroll
        for (int k = 0; k < Q; ++k) f[k] = __ldg(s + (k * plane - ey(k) * pitch - ex(k)));
    } else {
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            SrcSlot sl = stream_source(nx, ny, i, j, k, p.xper, p.yper, p.freeslip, p.halo_l, p.halo_r);
            f[k] = __ldg(p.src + p.L.at(sl.i, sl.j, sl.k));
        }
        // overrides by a select over the nine slots: an index known only at run time would put
        // f in local memory, and each load would then wait for the one before to be stored
        for (int q = 0; q < p.n_ovr; ++q)
            if (p.ovr[q].i == i && p.ovr[q].j == j) {
                const int kq = p.ovr[q].k;
                const T v = (T)p.ovr[q].v;
#pragma unroll
                for (int k = 0; k < Q; ++k) f[k] = k == kq ? v : f[k];
            }
    }
}

// Non-positive (or NaN) density at a node: set the handle's error flag.  The flag is read
// first, so a case that has gone unstable costs one atomic per SM until the flag is visible,
// not one per node and step on a single address.
template <class T>
__device__ __forceinline__ void flag_bad_density(const StepParams<T>& p) {
    if (__ldcg(p.errflag) == 0) atomicOr(p.errflag, 1);
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

// Field statistics: this step's post-closure u, v and p = rho cs2 (cs2 = 1/3, 2d_mrlbm.f90:153,
// 237) added to FP64 running sums of x and x^2.  Explicit round-to-nearest operations keep the
// sums free of contraction in every build, so they equal a host loop adding the same fields.
// The six old sums of a node are loaded (read-only path; each slot belongs to one thread of
// the launch) before the node's arithmetic, so their latency overlaps it.
struct FieldPre { double v[6]; };

template <class T>
__device__ __forceinline__ void fields_load(const StepParams<T>& p, int i, int j, FieldPre& q) {
    const int64_t n = (int64_t)(i - 1) + (int64_t)p.L.nx * (j - 1);
    const int64_t N = (int64_t)p.L.nx * p.L.ny;
#pragma unroll
    for (int c = 0; c < 6; ++c) q.v[c] = __ldg(p.fstat + n + c * N);
}

template <class T>
__device__ __forceinline__ void fields_store(const StepParams<T>& p, int i, int j, const FieldPre& q, double rho,
                                             double ux, double uy) {
    const int64_t n = (int64_t)(i - 1) + (int64_t)p.L.nx * (j - 1);
    const int64_t N = (int64_t)p.L.nx * p.L.ny;
    const double pr = __dmul_rn(rho, 1.0 / 3.0);
    double* a = p.fstat + n;
    a[0] = __dadd_rn(q.v[0], ux);
    a[N] = __dadd_rn(q.v[1], uy);
    a[2 * N] = __dadd_rn(q.v[2], pr);
    a[3 * N] = __dadd_rn(q.v[3], __dmul_rn(ux, ux));
    a[4 * N] = __dadd_rn(q.v[4], __dmul_rn(uy, uy));
    a[5 * N] = __dadd_rn(q.v[5], __dmul_rn(pr, pr));
}

template <class T>
__device__ __forceinline__ void accumulate_fields(const StepParams<T>& p, int i, int j, double rho, double ux,
                                                  double uy) {
    FieldPre q;
    fields_load(p, i, j, q);
    fields_store(p, i, j, q, rho, ux, uy);
}

// Body force (an extension: the reference has no forcing term).  A first-order momentum
// source added to the post-collision populations, fout_k += 3 w_k (c_k . g): it adds g to the
// node's momentum each step and leaves its mass unchanged.  Applied at bulk and edge nodes,
// not at curved-wall nodes.  In the FP32 form the same term is added to the deviations.
template <class T>
__device__ __forceinline__ void add_body_force(const StepParams<T>& p, int i, int j, T fo[Q]) {
    const int64_t n = (int64_t)(i - 1) + (int64_t)p.L.nx * (j - 1);
    const T fx = T(3) * p.body[n], fy = T(3) * p.body[(int64_t)p.L.nx * p.L.ny + n];
    const T w1 = p.w[1], w5 = p.w[5];
    fo[1] = fo[1] + w1 * fx;
    fo[3] = fo[3] - w1 * fx;
    fo[2] = fo[2] + w1 * fy;
    fo[4] = fo[4] - w1 * fy;
    fo[5] = fo[5] + w5 * (fx + fy);
    fo[7] = fo[7] - w5 * (fx + fy);
    fo[6] = fo[6] + w5 * (fy - fx);
    fo[8] = fo[8] - w5 * (fy - fx);
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
constexpr int AUX_CHUNK = 256;    // terms per warp and round in the in-order force sums

template <class T>
struct BTab {
    const T* g;
    const int* i;
    int n;                            // nodes per block (row stride of the staged tables)
    __device__ __forceinline__ T gf(int field, int li) const { return g[field * n + li]; }
    __device__ __forceinline__ int gi(int field, int li) const { return i[field * n + li]; }
};

// The per-step sums of the force record (Fx and Fy over the wall nodes, rho over the inlet
// column) are taken in index order, as the reference's sum() does (2d_mrlbm.f90:359,
// 488-489): the result does not depend on the launch shape and equals the reference's sums
// bit for bit.  Two tails do them, each in the last block of its group to finish: the last
// boundary block sums the forces (arrival counter 0), the last of the edge blocks that hold
// the inlet column sums rho (counter 1), so neither waits for the other group.

// True in the last of n blocks to arrive at counter c (block-uniform).
__device__ __forceinline__ bool last_to_arrive(unsigned* c, int n) {
    __shared__ unsigned ticket;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) ticket = atomicAdd(c, 1u);
    __syncthreads();
    const bool last = ticket == (unsigned)(n - 1);
    if (last) __threadfence();
    return last;
}

// ((0 + v[0]) + v[1]) + ... + v[n-1] by one warp, returned in lane 0.  The warp stages
// AUX_CHUNK terms per round in shared memory (st) with parallel loads and issues the next
// round's loads before lane 0 adds the current round, so only the adds are serial.
__device__ __forceinline__ double warp_ordered_sum(const double* v, int n, double* st, int lane) {
    constexpr int R = AUX_CHUNK / 32;
    double r[R];
#pragma unroll
    for (int u = 0; u < R; ++u) {
        const int q = u * 32 + lane;
        r[u] = q < n ? __ldcg(v + q) : 0.0;
    }
    double acc = 0.0;
    for (int q0 = 0; q0 < n; q0 += AUX_CHUNK) {
        const int m = min(AUX_CHUNK, n - q0);
#pragma unroll
        for (int u = 0; u < R; ++u) st[u * 32 + lane] = r[u];
        __syncwarp();
        const int q1 = q0 + AUX_CHUNK;
        if (q1 < n) {
#pragma unroll
            for (int u = 0; u < R; ++u) {
                const int q = q1 + u * 32 + lane;
                r[u] = q < n ? __ldcg(v + q) : 0.0;
            }
        }
        if (lane == 0) {
#pragma unroll 16
            for (int q = 0; q < m; ++q) acc = acc + st[q];
        }
        __syncwarp();
    }
    return acc;
}

// The record fields of a step: the launch's own, or for a replayed launch (p.call set) the ones
// its call state gives.
struct StepRec {
    int do_stats, iter;
    double* rec;
};
template <class T>
__device__ __forceinline__ StepRec step_rec(const StepParams<T>& p) {
    if (!p.call) return StepRec{p.do_stats, p.iter, p.rec};
    const int iter0 = __ldg(p.call), rn0 = __ldg(p.call + 1);
    StepRec r;
    r.iter = iter0 + p.bstep + 1;
    r.do_stats = r.iter >= p.stats_lo && r.iter <= p.stats_hi;
    const int before = max(0, min(r.iter - 1, p.stats_hi) - max(iter0 + 1, p.stats_lo) + 1);
    r.rec = r.do_stats ? p.ring + (size_t)(rn0 + before) * REC_WORDS : nullptr;
    return r;
}

// Force tail, called by every boundary block once its nodes' forces are in p.partials.
template <class Phys>
__device__ __forceinline__ void force_tail(const typename Phys::P& p, const StepRec& sr, unsigned char* smem) {
    if (!sr.do_stats) return;
    if (!last_to_arrive(p.counter, p.nbblk)) return;
    __shared__ double sm[2];
    const int tid = threadIdx.x, lane = tid & 31;
    for (int w = tid >> 5; w < 2; w += (int)(blockDim.x >> 5)) {     // Fx by warp 0, Fy by warp 1
        const double sum = warp_ordered_sum(p.partials + w * p.nb, p.nb, reinterpret_cast<double*>(smem) + w * AUX_CHUNK, lane);
        if (lane == 0) sm[w] = sum;
    }
    __syncthreads();
    if (tid == 0) {
        if (sr.rec) {
            sr.rec[0] = (double)sr.iter;
            sr.rec[1] = sm[0];
            sr.rec[2] = sm[1];
            if (p.halo_l) sr.rec[3] = 0.0;                  // an x-slab without column 1 adds 0
        }
        p.counter[0] = 0u;
    }
}

// The three sums of a force record, each over its terms in index order (one warp per sum):
// Fx over part[0, nb), Fy over part[nb, 2 nb), rho(1,j) over part[2 nb, 2 nb + ny) (0 on an
// x-slab without column 1).  Used for deferred records (the next launch sums the terms of the
// previous stats step) and by the finishing kernel; smem holds 3 * AUX_CHUNK doubles.
__device__ __forceinline__ void record_sums(const double* part, int nb, int ny, int halo_l, double* rec, int iter,
                                            unsigned char* smem) {
    const int tid = threadIdx.x, lane = tid & 31, nw = (int)(blockDim.x >> 5);
    double* st = reinterpret_cast<double*>(smem);
    for (int w = tid >> 5; w < 3; w += nw) {
        const int n = w < 2 ? nb : (halo_l ? 0 : ny);
        const double sum = warp_ordered_sum(part + w * nb, n, st + w * AUX_CHUNK, lane);
        if (lane == 0) rec[w + 1] = sum;
    }
    if (tid == 0) rec[0] = (double)iter;
}

// Edge blocks [0, inlet_blocks) hold the inlet column (it comes first in their enumeration).
__device__ __forceinline__ int inlet_blocks(int ny, int halo_l) {
    return halo_l ? 0 : (ny + (int)blockDim.x - 1) / (int)blockDim.x;
}

// Inlet tail, called by every edge block once its inlet nodes' rho are in p.partials.
template <class Phys>
__device__ __forceinline__ void inlet_tail(const typename Phys::P& p, const StepRec& sr, unsigned char* smem, int eb) {
    if (!sr.do_stats) return;
    const int nin = inlet_blocks(p.L.ny, p.halo_l);
    if (eb >= nin) return;
    if (!last_to_arrive(p.counter + 1, nin)) return;
    const int tid = threadIdx.x;
    if (tid < 32) {
        const double sum = warp_ordered_sum(p.partials + 2 * p.nb, p.L.ny, reinterpret_cast<double*>(smem), tid);
        if (tid == 0) {
            if (sr.rec) sr.rec[3] = sum;
            p.counter[1] = 0u;
        }
    }
}

// WIDE: the kernel has registers enough (Phys::WIDE_REGS per thread) for lane 0 to gather its
// node's own populations together with its stencil node's, and for the closure to be inlined.
// WAIT: the block itself waits for the previous step after staging its (creation-time) tables;
// otherwise the kernel waited before calling it.
template <class Phys, bool WIDE, bool WAIT>
__device__ __forceinline__ void boundary_block(const typename Phys::P& p, unsigned char* smem, int bb) {
    using T = typename Phys::T;
    T* sg = reinterpret_cast<T*>(smem);                               // G_STAGED * BNODES
    int* sgi = reinterpret_cast<int*>(smem + sizeof(T) * G_STAGED * BNODES);   // I_NFIELDS * BNODES
    const int nthr = blockDim.x, tid = threadIdx.x;
    const int bn = nthr / BLANES;
    const int l0 = bb * bn;
    // Every load of the staging is issued before the first shared-memory store, so the tables
    // arrive in one memory round trip instead of one per loop trip (after an L2 flush each trip
    // is a DRAM access, and the wall-node chain is on the step's critical path).  Each thread
    // stages G_STAGED / BLANES real and I_NFIELDS / BLANES integer entries (rounded up).
    {
        constexpr int GU = (G_STAGED + BLANES - 1) / BLANES, IU = (I_NFIELDS + BLANES - 1) / BLANES;
        T gv[GU];
        int iv[IU];
#pragma unroll
        for (int u = 0; u < GU; ++u) {
            const int idx = tid + u * nthr, f = idx / bn, n = idx - f * bn;
            gv[u] = (idx < G_STAGED * bn && l0 + n < p.nb) ? p.bgeo[f * p.nb + l0 + n] : T(0);
        }
#pragma unroll
        for (int u = 0; u < IU; ++u) {
            const int idx = tid + u * nthr, f = idx / bn, n = idx - f * bn;
            iv[u] = (idx < I_NFIELDS * bn && l0 + n < p.nb) ? p.bint[f * p.nb + l0 + n] : 0;
        }
#pragma unroll
        for (int u = 0; u < GU; ++u)
            if (tid + u * nthr < G_STAGED * bn) sg[tid + u * nthr] = gv[u];
#pragma unroll
        for (int u = 0; u < IU; ++u)
            if (tid + u * nthr < I_NFIELDS * bn) sgi[tid + u * nthr] = iv[u];
    }
    const StepRec sr = step_rec(p);
    const int li = tid / BLANES, lane = tid % BLANES;
    const int l = l0 + li;
    const bool active = l < p.nb;
    const bool interp = p.closure == CLOSURE_UNROTATED || p.vel_interp || p.mom_interp;
    const int r = lane >> 2, c = lane & 3;        // reference point 2 + r, corner c
    const int s = 4 * r + c;
    // this lane's stencil weights (creation-time tables, like the staged ones)
    T cc = T(0), ss = T(0), s2 = T(0);
    if (active && interp) {
        cc = p.bgeo[(G_SCC + s) * p.nb + l];
        ss = p.bgeo[(G_SSS + s) * p.nb + l];
        s2 = p.bgeo[(G_SS2 + s) * p.nb + l];
    }
    // The tables are written once, when the handle is created, so the staging above may run
    // while the previous step finishes; everything below reads or writes what steps change.
    if (WAIT) wait_prior_grid();
    __syncthreads();
    const BTab<T> tb{sg, sgi, bn};
    T fown[Q];
    if (WIDE && active && lane == 0) gather(p, tb.gi(I_NODEI, li), tb.gi(I_NODEJ, li), fown);
    T ux = T(0), uy = T(0), mx = T(0), my = T(0);
    const T xd = active ? tb.gf(r == 0 ? G_XD2 : G_XD3, li) : T(0);
    const T yd = active ? tb.gf(r == 0 ? G_YD2 : G_YD3, li) : T(0);
    if (active && interp) {
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
        if constexpr (WIDE) Phys::boundary_close_pre(p, tb, li, l, fown, ux, uy, mx, my, ux3, uy3, mx3, my3, Fx, Fy);
        else Phys::boundary_close(p, tb, li, l, ux, uy, mx, my, ux3, uy3, mx3, my3, Fx, Fy);
        if (sr.do_stats) { p.partials[l] = Fx; p.partials[p.nb + l] = Fy; }
    }
    if (!p.defer) force_tail<Phys>(p, sr, smem);
}

// Edge blocks: one thread per domain-edge node, so the edge closures (outlet neighbour gather,
// inlet/outlet/wall closures, 2d_mrlbm.f90:249-272, 313-351) run side by side instead of
// serially inside bulk tiles.  Order: column 1 (j = 1..ny), column nx, then rows 1 and ny
// without the corners; an x-slab's halo faces are not edges.  The thread of node (1,j) also
// records rho(1,j) after the closures for the inlet running mean (2d_mrlbm.f90:359).
template <class Phys>
__device__ __forceinline__ void edge_block(const typename Phys::P& p, int eb, unsigned char* smem) {
    const int nx = p.L.nx, ny = p.L.ny;
    const StepRec sr = step_rec(p);
    const int e = eb * (int)blockDim.x + (int)threadIdx.x;
    const int cl = p.halo_l ? 0 : 1, cr = p.halo_r ? 0 : 1;         // edge columns of this lattice
    const int nl = cl * ny, nr = cr * ny, nrow = nx - cl - cr;
    if (e < nl + nr + 2 * nrow) {
        int i, j;
        if (e < nl) { i = 1; j = e + 1; }
        else if (e < nl + nr) { i = nx; j = e - nl + 1; }
        else {
            const int q = e - nl - nr;
            i = cl + 1 + (q < nrow ? q : q - nrow);
            j = q < nrow ? 1 : ny;
        }
        const double rho = Phys::edge_bulk_node(p, i, j, CLS_FLUID);
        if (sr.do_stats && i == 1 && !p.halo_l) p.partials[2 * p.nb + j - 1] = rho;
    }
    if (!p.defer) inlet_tail<Phys>(p, sr, smem, eb);
    else if (eb == 0 && p.prev_rec) record_sums(p.prev_partials, p.nb, p.L.ny, p.halo_l, p.prev_rec, p.prev_iter, smem);
}

// Shared memory of an auxiliary block: the boundary tables and, afterwards, the tail's
// staged terms.
template <class T>
constexpr int aux_smem_bytes() {
    return (int)(sizeof(T) * G_STAGED + sizeof(int) * I_NFIELDS) * BNODES > 3 * AUX_CHUNK * (int)sizeof(double)
               ? (int)(sizeof(T) * G_STAGED + sizeof(int) * I_NFIELDS) * BNODES
               : 3 * AUX_CHUNK * (int)sizeof(double);
}

// Auxiliary work item b of a step: boundary block b (b < nbblk) or edge block b - nbblk.
template <class Phys, bool WIDE, bool WAIT = true>
__device__ __forceinline__ void aux_item(const typename Phys::P& p, unsigned char* smem, int b) {
    if (b < p.nbblk) boundary_block<Phys, WIDE, WAIT>(p, smem, b);
    else edge_block<Phys>(p, b - p.nbblk, smem);
}

// Whether a kernel of `threads` threads and `minb` resident blocks per SM takes the wide wall path.
template <class Phys>
constexpr bool wide_wall(int threads, int minb) { return 65536 / (threads * minb) >= Phys::WIDE_REGS; }

// ---- one time step as two launches ---------------------------------------------------------
// A step is an auxiliary launch (aux_kernel: the curved-wall boundary blocks, then the domain-edge
// blocks) followed by a bulk launch (every interior node by tiles of one shape); both write the
// next time level at disjoint nodes and read the previous one.  Each has its own register budget
// and instruction footprint, so the wall-node closures cost the bulk tiles nothing.  Ordering
// with programmatic dependent launch, per step n (A = auxiliary, B = bulk):
//   * A(n): every block waits for its predecessor in the stream (B(n-1), or whatever the caller
//     put in between) to complete, then allows B(n) to launch, then works;
//   * B(n): launches once every A(n) block has waited, hence after B(n-1) completed; it does
//     not wait itself, so its tiles run beside the wall-node chain.  It allows the next launch
//     (A(n+1)) at once, and the last of its blocks to finish waits for A(n) to complete, so
//     B(n) completes only after A(n): whatever follows B(n) in the stream sees the whole step.
constexpr int AUX_THREADS = 128;

template <class Phys>
__global__ void __launch_bounds__(AUX_THREADS) aux_kernel(const __grid_constant__ typename Phys::P p) {
    __shared__ __align__(16) unsigned char smem[aux_smem_bytes<typename Phys::T>()];
    wait_prior_grid();
    aux_item<Phys, true, false>(p, smem, (int)blockIdx.x);
}

// Start of a bulk launch: let the next launch (the next step's auxiliary blocks) be scheduled.
__device__ __forceinline__ void bulk_begin() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// End of a bulk block: the last block of the launch to get here waits for the step's auxiliary
// launch to complete (counter[2] counts the bulk blocks; the last one resets it).
template <class T>
__device__ __forceinline__ void bulk_end(const StepParams<T>& p) {
    if (threadIdx.x == 0 && atomicAdd(p.counter + 2, 1u) == gridDim.x - 1) {
        p.counter[2] = 0u;
        asm volatile("griddepcontrol.wait;" ::: "memory");
    }
}


template <class P>
inline int edge_blocks(const P& p, int nthr) {
    const int n = 2 * p.L.nx + (p.halo_l ? 0 : p.L.ny - 2) + (p.halo_r ? 0 : p.L.ny - 2);
    return (n + nthr - 1) / nthr;
}

template <class Phys>
inline int launch_aux(typename Phys::P p, cudaStream_t s) {
    const int bn = AUX_THREADS / BLANES;
    p.nbblk = p.nb > 0 ? (p.nb + bn - 1) / bn : 1;
    p.neblk = edge_blocks(p, AUX_THREADS);
    return launch_after_prior(aux_kernel<Phys>, (unsigned)(p.nbblk + p.neblk), AUX_THREADS, 0, s, p) == cudaSuccess ? 0 : -1;
}

// True when every node of columns i0..i1 and rows j0..j1 is an interior bulk node: no domain
// edge (an x-slab's halo faces are not edges), nothing beyond the lattice, no node of the
// cylinder's bounding box.  Block-uniform when the bounds are.
template <class T>
__device__ __forceinline__ bool plain_tile(const StepParams<T>& p, int i0, int i1, int j0, int j1) {
    return col_interior(p, i0) && i1 <= p.L.nx && col_interior(p, i1) && j0 > 1 && j1 < p.L.ny &&
           (i1 < p.box_x0 || i0 >= p.box_x0 + p.box_w || j1 < p.box_y0 || j0 >= p.box_y0 + p.box_h);
}

// Interior populations (no wraps, no ghosts): the branch-free half of `gather`.
template <class T>
__device__ __forceinline__ void gather_interior(const StepParams<T>& p, int i, int j, T f[Q]) {
    const int pitch = p.L.pitch, plane = (int)p.L.plane;
    const T* s = p.src + ((int)(j * pitch + i + p.L.off));
#pragma unroll
    for (int k = 0; k < Q; ++k) f[k] = __ldg(s + (k * plane - ey(k) * pitch - ex(k)));
}

// Tile t's column and row of tiles, by a multiply-high where the launcher provided one.
template <class T>
__device__ __forceinline__ void tile_coords(const StepParams<T>& p, int t, int& tx, int& ty) {
    ty = p.tx_magic ? (int)(((unsigned long long)(unsigned)t * p.tx_magic) >> 32) : t / p.tiles_x;
    tx = t - ty * p.tiles_x;
}

// Bulk tiles of BX x (BY*NJ) nodes, one thread per column and NJ rows, one tile per block.  A
// thread first issues the loads of all its interior rows, then finishes them (collide and store)
// one by one, so up to 9*NJ loads per thread are in flight.
template <class Phys, int BX, int BY, int NJ>
__device__ __forceinline__ void tile_body(const typename Phys::P& p, int t) {
    using T = typename Phys::T;
    int tx, ty;
    tile_coords(p, t, tx, ty);
    const int lx = threadIdx.x % BX, ly = threadIdx.x / BX;
    const int i = 1 + tx * BX + lx;
    const int nx = p.L.nx, ny = p.L.ny;
    if (plain_tile(p, 1 + tx * BX, 1 + tx * BX + BX - 1, 1 + ty * BY * NJ, ty * BY * NJ + BY * NJ)) {
        // no edge, ghost or cylinder-box node in the tile: no per-node class or edge tests
        T f[NJ][Q];
#pragma unroll
        for (int r = 0; r < NJ; ++r) gather_interior(p, i, 1 + ty * BY * NJ + r * BY + ly, f[r]);
#pragma unroll
        for (int r = 0; r < NJ; ++r) Phys::finish(p, i, 1 + ty * BY * NJ + r * BY + ly, CLS_FLUID, f[r]);
        return;
    }
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
            if (cls[r] == CLS_SOLID && p.call && p.plot_every > 0 &&
                (__ldg(p.call) + p.bstep + 1) % p.plot_every == 0)
                cls[r] = CLS_SOLID_ZERO;                      // a replayed launch's plot step
            if (cls[r] < 0 && is_interior(p, i, j)) {
                gather_interior(p, i, j, f[r]);
                interior |= 1u << r;
            }
        }
    }
#pragma unroll
    for (int r = 0; r < NJ; ++r) {
        const int j = 1 + ty * BY * NJ + r * BY + ly;
        if ((interior >> r) & 1u) Phys::finish(p, i, j, cls[r], f[r]);    // edge nodes: edge blocks
    }
}

template <class Phys, int BX, int BY, int NJ, int MINB>
__global__ void __launch_bounds__(BX * BY, MINB) step_kernel(const __grid_constant__ typename Phys::P p) {
    bulk_begin();
    tile_body<Phys, BX, BY, NJ>(p, (int)blockIdx.x);
    bulk_end(p);
}

// ---- 128-bit vector bulk path -------------------------------------------------------------
// Each lane owns VW consecutive nodes of a row (VW = 16 bytes / element: four FP32 or two FP64
// nodes) and reads every direction plane with one aligned 16-byte load per plane.  A pull
// source one column left (planes with e_kx = +1) or right (e_kx = -1) of the lane's group comes
// from the neighbouring lane by a warp shuffle; the warp's two outermost lanes (and, in an
// x-slab, the lane ending at column nx) fetch that column with one scalar load.  A group whose nodes are all interior bulk nodes is written
// back with one 16-byte store per plane; groups touching an edge or the cylinder box fall back
// to per-node handling (edge nodes belong to the edge blocks, wall nodes to the boundary
// blocks).  Columns read: i0-1 .. i0+VW of rows j-1 .. j+1, which the layout's row slack
// (pitch >= off + nx + 4) keeps inside the row for every group with i0 <= nx.
template <class T> struct Vec16;
template <> struct Vec16<float> {
    static constexpr int N = 4;
    static __device__ __forceinline__ void load(const float* a, float (&v)[4]) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(a));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    }
    static __device__ __forceinline__ void store(float* a, const float (&v)[4]) {
        *reinterpret_cast<float4*>(a) = make_float4(v[0], v[1], v[2], v[3]);
    }
};
template <> struct Vec16<double> {
    static constexpr int N = 2;
    static __device__ __forceinline__ void load(const double* a, double (&v)[2]) {
        const double2 t = __ldg(reinterpret_cast<const double2*>(a));
        v[0] = t.x; v[1] = t.y;
    }
    static __device__ __forceinline__ void store(double* a, const double (&v)[2]) {
        *reinterpret_cast<double2*>(a) = make_double2(v[0], v[1]);
    }
};

template <class Phys, int WARPS, int NJ>
__device__ __forceinline__ void vec_tile(const typename Phys::P& p, int t) {
    using T = typename Phys::T;
    using VT = Vec16<T>;
    constexpr int VW = VT::N;
    int tx, ty;
    tile_coords(p, t, tx, ty);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nx = p.L.nx, ny = p.L.ny;
    const int i0 = 1 + (tx * 32 + lane) * VW;
    const bool act = i0 <= nx;
    const int pitch = p.L.pitch, plane = (int)p.L.plane;
    // cylinder-box overlap of this lane's columns (rows checked per row)
    const bool box_cols = (i0 + VW - 1 >= p.box_x0) && (i0 < p.box_x0 + p.box_w);
#pragma unroll 1
    for (int r = 0; r < NJ; ++r) {
        const int j = 1 + (ty * WARPS + warp) * NJ + r;
        if (j > ny) break;                                    // uniform across the warp
        T v[Q][VW];
        T side[Q];                                            // column i0-1 (e_kx=+1) or i0+VW (e_kx=-1)
        const int rowbase = j * pitch + i0 + p.L.off;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            const T* a = p.src + (rowbase + k * plane - ey(k) * pitch);
            if (act) VT::load(a, v[k]);
            else {
#pragma unroll
                for (int n = 0; n < VW; ++n) v[k][n] = T(0);
            }
            if (ex(k) > 0) {
                side[k] = __shfl_up_sync(0xffffffffu, v[k][VW - 1], 1);
                if (lane == 0 && act) side[k] = __ldg(a - 1);
            } else if (ex(k) < 0) {
                side[k] = __shfl_down_sync(0xffffffffu, v[k][0], 1);
                // the warp's last lane, and the lane whose group ends at node nx of an x-slab
                // (its right neighbour's column nx+1 is the halo, which no lane loads)
                if ((lane == 31 && i0 + VW <= nx) || (p.halo_r && act && i0 + VW - 1 == nx))
                    side[k] = __ldg(a + VW);
            }
        }
        if (!act) continue;
        const bool row_int = j > 1 && j < ny;
        const bool in_box_row = box_cols && (unsigned)(j - p.box_y0) < (unsigned)p.box_h;
        const bool all_int = row_int && col_interior(p, i0) && i0 + VW - 1 <= nx && col_interior(p, i0 + VW - 1) &&
                             !in_box_row;
        T out[Q][VW];
#pragma unroll
        for (int n = 0; n < VW; ++n) {
            const int i = i0 + n;
            T f[Q];
#pragma unroll
            for (int k = 0; k < Q; ++k) {
                if (ex(k) == 0) f[k] = v[k][n];
                else if (ex(k) > 0) f[k] = n == 0 ? side[k] : v[k][n - 1];
                else f[k] = n == VW - 1 ? side[k] : v[k][n + 1];
            }
            if (all_int) {
                T fo[Q];
                Phys::compute(p, i, j, CLS_FLUID, f, fo);
#pragma unroll
                for (int k = 0; k < Q; ++k) out[k][n] = fo[k];
            } else if (row_int && i <= nx && col_interior(p, i)) {   // edge nodes: edge blocks
                const int cls = in_box_row ? node_class(p, i, j) : CLS_FLUID;
                if (cls < 0) Phys::finish(p, i, j, cls, f);   // cls >= 0: curved-wall node
            }
        }
        if (all_int) {
            T* d = p.dst + rowbase;
#pragma unroll
            for (int k = 0; k < Q; ++k) VT::store(d + k * plane, out[k]);
        }
    }
}

template <class Phys, int WARPS, int NJ, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) step_kernel_vec(const __grid_constant__ typename Phys::P p) {
    bulk_begin();
    vec_tile<Phys, WARPS, NJ>(p, (int)blockIdx.x);
    bulk_end(p);
}

template <class Phys, int WARPS, int NJ, int MINB>
int launch_step_vec(typename Phys::P p, cudaStream_t s) {
    using T = typename Phys::T;
    constexpr int VW = Vec16<T>::N;
    const int nthr = WARPS * 32;
    if (launch_aux<Phys>(p, s) != 0) return -1;
    p.nbblk = p.neblk = 0;
    p.tiles_x = (p.L.nx + 32 * VW - 1) / (32 * VW);
    const int tiles_y = (p.L.ny + WARPS * NJ - 1) / (WARPS * NJ);
    const long long nblocks = (long long)p.tiles_x * tiles_y;
    p.tx_magic = tile_div_magic(p.tiles_x, nblocks);
    return launch_after_prior(step_kernel_vec<Phys, WARPS, NJ, MINB>, (unsigned)nblocks, nthr, 0, s, p) == cudaSuccess ? 0
                                                                                                            : -1;
}

// ---- persistent software-pipelined bulk path -------------------------------------------------
// A fixed grid of resident blocks walks the row segments of the lattice (segment u: row
// 1 + u / tiles_x, columns (u % tiles_x) * B + 1 ..) with a stride of the grid size.  Each
// thread loads the populations of its next node before it collides and stores the current
// one, so a load is always in flight behind the arithmetic and no block waits out a tail
// wave.  Edge and wall nodes are skipped (edge and boundary blocks own them).
template <class Phys, int B>
__device__ __forceinline__ void pipe_body(const typename Phys::P& p) {
    using T = typename Phys::T;
    const int nx = p.L.nx, ny = p.L.ny, tiles_x = p.tiles_x;
    const int units = tiles_x * ny;
    const int G = (int)gridDim.x;
    auto fetch = [&](int u, T (&f)[Q], int& i, int& j) -> bool {
        if (u >= units) return false;
        j = 1 + u / tiles_x;
        i = 1 + (u - (j - 1) * tiles_x) * B + (int)threadIdx.x;
        if (!(i <= nx && is_interior(p, i, j))) return false;
        gather_interior(p, i, j, f);
        return true;
    };
    int u = (int)blockIdx.x;
    T a[Q], b[Q];
    int ia = 0, ja = 0, ib = 0, jb = 0;
    bool va = fetch(u, a, ia, ja);
    while (u < units) {
        const int un = u + G;
        const bool vb = fetch(un, b, ib, jb);
        if (va) {
            const int cls = node_class(p, ia, ja);
            if (cls < 0) Phys::finish(p, ia, ja, cls, a);     // cls >= 0: curved-wall node
        }
#pragma unroll
        for (int k = 0; k < Q; ++k) a[k] = b[k];
        ia = ib;
        ja = jb;
        va = vb;
        u = un;
    }
}

template <class Phys, int B, int MINB>
__global__ void __launch_bounds__(B, MINB) step_kernel_pipe(const __grid_constant__ typename Phys::P p) {
    bulk_begin();
    pipe_body<Phys, B>(p);
    bulk_end(p);
}

template <class Phys, int B, int MINB>
int launch_step_pipe(typename Phys::P p, cudaStream_t s) {
    static int per_sm[64] = {0}, sms[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64) return -1;
    if (!per_sm[dev]) {
        if (cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[dev], step_kernel_pipe<Phys, B, MINB>, B, 0) !=
                cudaSuccess || per_sm[dev] <= 0)
            return -1;
    }
    if (launch_aux<Phys>(p, s) != 0) return -1;
    p.nbblk = p.neblk = 0;
    p.tiles_x = (p.L.nx + B - 1) / B;
    const long long units = (long long)p.tiles_x * p.L.ny;
    const long long G = std::min<long long>(units, (long long)sms[dev] * per_sm[dev]);
    return launch_after_prior(step_kernel_pipe<Phys, B, MINB>, (unsigned)G, B, 0, s, p) == cudaSuccess ? 0 : -1;
}

// Halo faces of an x-slab, ahead of the step: one thread per node of column 1 (left halo
// face) and column nx (right halo face), computing the node exactly as the step kernel does
// and writing it into the next time level.  The step kernel then writes the same bits again;
// in between, the populations that cross the faces can already travel to the neighbours
// while the rest of the slab is computed.  The caller clears fstat and macro (the step
// kernel accumulates them) and do_stats.  A face never holds a wall node: the partition
// keeps the cylinder and its stencils inside one slab.
template <class Phys>
__global__ void __launch_bounds__(128) face_kernel(const __grid_constant__ typename Phys::P p) {
    using T = typename Phys::T;
    wait_prior_grid();
    const int ny = p.L.ny;
    const int n = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (n >= 2 * ny) return;
    const int side = n / ny, j = 1 + (n - side * ny);
    if (side == 0 ? !p.halo_l : !p.halo_r) return;
    const int i = side == 0 ? 1 : p.L.nx;
    if (j == 1 || j == ny) {                          // rows 1 and ny: edge nodes
        Phys::edge_bulk_node(p, i, j, CLS_FLUID);
        return;
    }
    const int cls = node_class(p, i, j);
    if (cls >= 0) return;
    T f[Q];
    gather(p, i, j, f);
    Phys::finish(p, i, j, cls, f);
}

template <class Phys>
int launch_face(const typename Phys::P& p, cudaStream_t s) {
    const int n = 2 * p.L.ny;
    return launch_after_prior(face_kernel<Phys>, (unsigned)((n + 127) / 128), 128, 0, s, p) == cudaSuccess ? 0 : -1;
}

// One launch for the whole step (Phys::FUSED_AUX): blocks [0, nbblk) are wall blocks of BX*BY/8
// nodes, the next neblk edge blocks of BX*BY nodes, then the bulk tiles; every block waits for
// the previous step first (the wall blocks after staging their tables), so no block of the
// step needs to wait for another launch.
template <class Phys, int BX, int BY, int NJ, int MINB>
__global__ void __launch_bounds__(BX * BY, MINB) step_kernel_fused(const __grid_constant__ typename Phys::P p) {
    __shared__ __align__(16) unsigned char smem[aux_smem_bytes<typename Phys::T>()];
    const int b = (int)blockIdx.x;
    if (b < p.nbblk) {
        boundary_block<Phys, wide_wall<Phys>(BX * BY, MINB), true>(p, smem, b);
        return;
    }
    wait_prior_grid();
    if (b < p.nbblk + p.neblk) edge_block<Phys>(p, b - p.nbblk, smem);
    else tile_body<Phys, BX, BY, NJ>(p, b - p.nbblk - p.neblk);
}

template <class Phys, int BX, int BY, int NJ, int MINB>
int launch_step_tiles(typename Phys::P p, cudaStream_t s) {
    const int nthr = BX * BY;
    p.tiles_x = (p.L.nx + BX - 1) / BX;
    const int tiles_y = (p.L.ny + BY * NJ - 1) / (BY * NJ);
    const long long nblocks = (long long)p.tiles_x * tiles_y;
    p.tx_magic = tile_div_magic(p.tiles_x, nblocks);
    if constexpr (Phys::FUSED_AUX) {
        const int bn = nthr / BLANES;
        p.nbblk = p.nb > 0 ? (p.nb + bn - 1) / bn : 1;
        p.neblk = edge_blocks(p, nthr);
        return launch_after_prior(step_kernel_fused<Phys, BX, BY, NJ, MINB>, (unsigned)(p.nbblk + p.neblk + nblocks), nthr,
                                  0, s, p) == cudaSuccess
                   ? 0
                   : -1;
    }
    if (launch_aux<Phys>(p, s) != 0) return -1;
    p.nbblk = p.neblk = 0;
    return launch_after_prior(step_kernel<Phys, BX, BY, NJ, MINB>, (unsigned)nblocks, nthr, 0, s, p) == cudaSuccess ? 0 : -1;
}

}  // namespace mrlbm
