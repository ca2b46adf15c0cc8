// surface.cuh -- surface pressure on the cylinder, its Gaussian smoothing over theta, and the
// four wake probes (write_statistics_out / extrapolate_var_on_cylinder / gaussian_smoothing /
// quadratic_interpolation, 2d_mrlbm.f90:593-766, and the probe records, 2d_mrlbm.f90:462-476).
//
// Runs after a statistics step on the populations that step gathered, so it sees the field
// the reference's p = rho cs2 is computed from (2d_mrlbm.f90:236; p is not updated by the
// boundary closures).  Kernel A (one block): per wall node, p at the bilinear stencils of
// reference points 2, 3 and 4, quadratic extrapolation in r to the wall point, reordered by
// theta; the probes.  Kernel B: the smoothing, p_fit(i) = sum_j W(i,j) ps(j) / sum_j W(i,j), with
// the weights exp(-(theta_i - theta_j)^2 / (2 sigma^2)) (sigma = 0.1) computed once on the
// host with the same libm the reference uses.  Every sum runs in the reference's index order.
#pragma once
#include "surface.h"
#include "step_fp64.cuh"

namespace mrlbm {
namespace surf {

// Populations of node (i, j) as the reference's f (FP64; FP32 storage adds back w_k).
template <class T>
__device__ __forceinline__ void gather_f(const StepParams<T>& p, int i, int j, double f[Q]) {
    T g[Q];
    gather(p, i, j, g);
#pragma unroll
    for (int k = 0; k < Q; ++k) f[k] = sizeof(T) == 8 ? (double)g[k] : (double)p.w[k] + (double)g[k];
}

template <class T>
__device__ __forceinline__ double node_p(const StepParams<T>& p, int i, int j) {
    double f[Q];
    gather_f(p, i, j, f);
    double s = f[0];
    s = s + f[1]; s = s + f[2]; s = s + f[3]; s = s + f[4];
    s = s + f[5]; s = s + f[6]; s = s + f[7]; s = s + f[8];
    return s * (1.0 / 3.0);                       // p = rho * cs2, cs2 = 1.0d0/3.0d0
}

template <class T>
__global__ void __launch_bounds__(256) surface_a(const __grid_constant__ StepParams<T> p, const __grid_constant__ SurfaceTables t,
                                                 double* rec, double* prec) {
    extern __shared__ double pcy[];               // [nb]
    const int nb = t.nb;
    for (int l = threadIdx.x; l < nb; l += blockDim.x) {
        double var[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) {             // reference points 2, 3, 4
            const int b = 4 * r;
            const double p1 = node_p(p, __ldg(p.bint + (I_SI + b + 0) * nb + l), __ldg(p.bint + (I_SJ + b + 0) * nb + l));
            const double p2 = node_p(p, __ldg(p.bint + (I_SI + b + 1) * nb + l), __ldg(p.bint + (I_SJ + b + 1) * nb + l));
            const double p3 = node_p(p, __ldg(p.bint + (I_SI + b + 2) * nb + l), __ldg(p.bint + (I_SJ + b + 2) * nb + l));
            const double p4 = node_p(p, __ldg(p.bint + (I_SI + b + 3) * nb + l), __ldg(p.bint + (I_SJ + b + 3) * nb + l));
            const double xd = (double)__ldg(p.bgeo + (G_XD2 + 2 * r) * nb + l);
            const double yd = (double)__ldg(p.bgeo + (G_YD2 + 2 * r) * nb + l);
            const double v0 = (1.0 - xd) * p1 + xd * p2;
            const double v1 = (1.0 - xd) * p3 + xd * p4;
            var[r] = (1.0 - yd) * v0 + yd * v1;
        }
        // quadratic_interpolation(x2,y2,var2, x3,y3,var3, x4,y4,var4, xs,ys): its (r1, r2, r3)
        // are the radii of points 2, 3, 4 and rs that of the wall point
        const double r1 = t.quad[5 * l], r2 = t.quad[5 * l + 1], r3 = t.quad[5 * l + 2];
        const double rs = t.quad[5 * l + 3], denom = t.quad[5 * l + 4];
        const double q1 = var[0], q2 = var[1], q3 = var[2];
        const double a0 = (r1 * r3 * q2 * (r3 - r1) + (r2 * r2) * (r3 * q1 - r1 * q3) + r2 * ((r1 * r1) * q3 - (r3 * r3) * q1)) / denom;
        const double a1 = ((r3 * r3) * (q1 - q2) + (r1 * r1) * (q2 - q3) + (r2 * r2) * (q3 - q1)) / denom;
        const double a2 = (r3 * (q2 - q1) + r2 * (q1 - q3) + r1 * (q3 - q2)) / denom;
        pcy[l] = a0 + a1 * rs + a2 * (rs * rs);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nb; k += blockDim.x) rec[k] = pcy[__ldg(t.idx + k)];
    if (threadIdx.x < 4 && prec) {
        const int i = t.probe_i[threadIdx.x], j = t.probe_j[threadIdx.x];
        double f[Q];
        gather_f(p, i, j, f);
        double rho, ux, uy;
        if (sizeof(T) == 8 && !is_interior(p, i, j)) {
            const fp64::Mac m = fp64::node_macro(reinterpret_cast<const StepParams<double>&>(p), i, j, f);
            rho = m.rho; ux = m.ux; uy = m.uy;
        } else {
            fp64::moments_u(f, rho, ux, uy);
        }
        prec[threadIdx.x] = rho / 3.0;             // 2d_mrlbm.f90:470-475: rho/3, ux/3, uy/3
        prec[4 + threadIdx.x] = ux / 3.0;
        prec[8 + threadIdx.x] = uy / 3.0;
    }
}

__global__ void surface_b(const __grid_constant__ SurfaceTables t, double* rec) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.nb) return;
    const double* ps = rec;
    double s = 0.0;
    for (int j = 0; j < t.nb; ++j) s = s + __ldg(t.W + (size_t)j * t.nb + i) * ps[j];
    rec[t.nb + i] = s / __ldg(t.sumw + i);
}

template <class T>
int launch_surface(const StepParams<T>& p, const SurfaceTables& t, double* rec, double* prec, cudaStream_t s) {
    if (t.nb <= 0) return 0;
    const size_t smem = (size_t)t.nb * sizeof(double);
    if (smem > 48 * 1024) return -2;
    surface_a<T><<<1, 256, smem, s>>>(p, t, rec, prec);
    surface_b<<<(t.nb + 127) / 128, 128, 0, s>>>(t, rec);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace surf
}  // namespace mrlbm
