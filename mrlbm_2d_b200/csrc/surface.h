// surface.h -- host interface of the surface-pressure and probe kernels (surface.cuh).
#pragma once
#include <cuda_runtime.h>
#include "step_params.h"

namespace mrlbm {

// Per-case constant tables of the surface output.
struct SurfaceTables {
    const double* quad;     // [5 * nb] per wall node: r(point 2), r(point 3), r(point 4), r(point 1), denom
    const int* idx;         // [nb] wall-node order by increasing theta (2d_mrlbm.f90:1138-1156)
    const double* W;        // [nb * nb] Gaussian weights, W[j * nb + i] (column j contiguous over i)
    const double* sumw;     // [nb] sum_j W[j * nb + i] in index order
    int probe_i[4], probe_j[4];
    int nb;
};

// One statistics step's surface pressure (sorted by theta) into rec[0 .. nb), its Gaussian
// smoothing into rec[nb .. 2 nb) and the probes' rho/3, ux/3, uy/3 into prec[0 .. 12), from
// the populations the step gathered (p.src).  FP64 arithmetic in the reference's order.
int launch_surface_f64(const StepParams<double>& p, const SurfaceTables& t, double* rec, double* prec, cudaStream_t s);
int launch_surface_f32(const StepParams<float>& p, const SurfaceTables& t, double* rec, double* prec, cudaStream_t s);

}  // namespace mrlbm
