// adjoint.h -- host interface of the adjoint step kernels (adjoint.cuh, launched from step_f64.cu).
#pragma once
#include <cuda_runtime.h>
#include "step_params.h"

namespace mrlbm {
namespace adj {

struct AdjArgs {
    double* lam_in;            // lambda^n = dJ/dF^n, padded layout; cleared as it is read
    double* lam_out;           // lambda^{n-1}, padded layout, zeroed before the step
    double* grad_body;         // [2 N] accumulated dJ/d(body force), or null
    double* grad_uin;          // [ny] accumulated dJ/d(u_in), or null
    double wJ;                 // weight of this step's drag in J (1/T inside the window, else 0)
    int n_edge;                // edge nodes: 2 ny (columns 1 and nx), + 2 (nx - 2) with no-slip reference walls
    unsigned* done;            // bulk blocks of the step's bulk launch that have finished (zero between steps)
    // Bounding box of the curved-wall stencil nodes (empty: sx0 > sx1).  A slot of lambda^{n-1}
    // is pulled by one node only, except the slots a stencil node pulls (its wall node reads them
    // too) and those of column nx - 1 (the outlet copies them): bulk nodes inside the box or in
    // that column add atomically, every other interior node stores its nine slots outright.
    int sx0, sx1, sy0, sy1;
};

}  // namespace adj

// One adjoint step: p describes forward step n (src = F^{n-1}); lambda^{n-1} must be zero.
// The step reads every in-domain slot of lambda^n exactly once and leaves it zero, so the two
// adjoint buffers alternate without clearing.
// FP32 handles: the forward states are FP32 deviations, the adjoint arithmetic is FP64.
int launch_adjoint_step(const StepParams<double>& p, const adj::AdjArgs& a, cudaStream_t s);
int launch_adjoint_step(const StepParams<float>& p, const adj::AdjArgs& a, cudaStream_t s);

}  // namespace mrlbm
