// state_io.cu -- device-side layout conversion for mrlbm_load_state / mrlbm_get_state /
// mrlbm_step_noalloc: one bulk host<->device copy plus a kernel instead of a host loop.
#include <algorithm>
#include "state_io.h"

namespace mrlbm {

namespace {

__device__ __forceinline__ double weight(int k, double w0, double w1, double w5) { return k == 0 ? w0 : (k < 5 ? w1 : w5); }

template <class T>
__global__ void scatter_state(const double* __restrict__ f0, T* a, T* b, Layout L, int xper, int yper, int freeslip,
                              double w0, double w1, double w5, int deviation, int hl, int hr) {
    const int64_t N = (int64_t)L.nx * L.ny;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N * Q) return;
    const int k = (int)(t / N);
    const int64_t n = t - (int64_t)k * N;
    const int i = (int)(n % L.nx) + 1, j = (int)(n / L.nx) + 1;
    const SrcSlot s = stream_source(L.nx, L.ny, i, j, k, xper != 0, yper != 0, freeslip != 0, hl != 0, hr != 0);
    const int64_t slot = L.at(s.i, s.j, s.k);
    const T v = deviation ? (T)(f0[t] - weight(k, w0, w1, w5)) : (T)f0[t];
    a[slot] = v;
    if (b) b[slot] = v;
}

template <class T>
__global__ void gather_state(const T* __restrict__ src, double* f, Layout L, int xper, int yper, int freeslip,
                             double w0, double w1, double w5, int deviation, int hl, int hr) {
    const int64_t N = (int64_t)L.nx * L.ny;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N * Q) return;
    const int k = (int)(t / N);
    const int64_t n = t - (int64_t)k * N;
    const int i = (int)(n % L.nx) + 1, j = (int)(n / L.nx) + 1;
    const SrcSlot s = stream_source(L.nx, L.ny, i, j, k, xper != 0, yper != 0, freeslip != 0, hl != 0, hr != 0);
    const double v = (double)src[L.at(s.i, s.j, s.k)];
    f[t] = deviation ? weight(k, w0, w1, w5) + v : v;
}

template <class T>
__global__ void fill_overrides(const double* __restrict__ f0, OvrEntry* ovr, int n, int nx, int ny, double w0,
                               double w1, double w5, int deviation) {
    const int q = threadIdx.x;
    if (q >= n) return;
    const OvrEntry e = ovr[q];
    const double v = f0[(int64_t)(e.i - 1) + (int64_t)nx * (e.j - 1) + (int64_t)nx * ny * e.k];
    ovr[q].v = deviation ? (double)(T)(v - weight(e.k, w0, w1, w5)) : v;
}

unsigned blocks_for(const Layout& L) { return (unsigned)(((int64_t)L.nx * L.ny * Q + 255) / 256); }

}  // namespace

cudaError_t launch_scatter_state(int precision, const double* f0, void* a, void* b, const Layout& L, int xper,
                                 int yper, int freeslip, const double* w, cudaStream_t s, int hl, int hr) {
    if (precision == 64)
        scatter_state<double><<<blocks_for(L), 256, 0, s>>>(f0, (double*)a, (double*)b, L, xper, yper, freeslip, w[0],
                                                            w[1], w[5], 0, hl, hr);
    else
        scatter_state<float><<<blocks_for(L), 256, 0, s>>>(f0, (float*)a, (float*)b, L, xper, yper, freeslip, w[0], w[1],
                                                           w[5], 1, hl, hr);
    return cudaGetLastError();
}

cudaError_t launch_gather_state(int precision, const void* src, double* f, const Layout& L, int xper, int yper,
                                int freeslip, const double* w, cudaStream_t s, int hl, int hr) {
    if (precision == 64)
        gather_state<double><<<blocks_for(L), 256, 0, s>>>((const double*)src, f, L, xper, yper, freeslip, w[0], w[1],
                                                           w[5], 0, hl, hr);
    else
        gather_state<float><<<blocks_for(L), 256, 0, s>>>((const float*)src, f, L, xper, yper, freeslip, w[0], w[1],
                                                          w[5], 1, hl, hr);
    return cudaGetLastError();
}

cudaError_t launch_fill_overrides(int precision, const double* f0, OvrEntry* ovr, int n, int nx, int ny,
                                  const double* w, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (precision == 64)
        fill_overrides<double><<<1, 64, 0, s>>>(f0, ovr, n, nx, ny, w[0], w[1], w[5], 0);
    else
        fill_overrides<float><<<1, 64, 0, s>>>(f0, ovr, n, nx, ny, w[0], w[1], w[5], 1);
    return cudaGetLastError();
}

namespace {
__global__ void field_stats_finalize(const double* __restrict__ sums, double* __restrict__ out, int64_t N, double n) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double mean = __ddiv_rn(sums[c * N + q], n);
            const double var = __dadd_rn(__ddiv_rn(sums[(3 + c) * N + q], n), -__dmul_rn(mean, mean));
            out[c * N + q] = mean;
            out[(3 + c) * N + q] = __dsqrt_rn(var > 0.0 ? var : 0.0);
        }
    }
}
}  // namespace

cudaError_t launch_field_stats_finalize(const double* sums, double* out, int64_t N, int64_t n, cudaStream_t s) {
    const int64_t blocks = std::min<int64_t>((N + 255) / 256, 148 * 16);
    field_stats_finalize<<<(unsigned)blocks, 256, 0, s>>>(sums, out, N, (double)n);
    return cudaGetLastError();
}

}  // namespace mrlbm
