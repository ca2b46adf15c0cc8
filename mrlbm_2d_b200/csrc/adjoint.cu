// adjoint.cu -- adjoint step instantiations.  Unlike the forward step units this one lets the
// compiler contract multiply-adds: the adjoint's arithmetic only has to be accurate, not to
// round like the reference, and contraction shortens the dual-number chains of the wall and
// edge maps.
#include "adjoint.cuh"

namespace mrlbm {

// One adjoint step: the wall and edge-column blocks, then the bulk blocks (adjoint.cuh).
template <class T>
static int launch_adjoint(const StepParams<T>& p, const adj::AdjArgs& a, cudaStream_t s) {
    const int64_t nodes = (int64_t)p.L.nx * p.L.ny;
    const int64_t aux = (int64_t)p.nb + (a.n_edge + 6) / 7;
    cudaError_t e;
    switch (p.closure) {                               // the curved-wall closure, one instantiation each
    case CLOSURE_STRONG: e = launch_after_prior(adj::adjoint_aux<StepParams<T>, CLOSURE_STRONG>, (unsigned)aux, 128, 0, s, p, a); break;
    case CLOSURE_WEAK: e = launch_after_prior(adj::adjoint_aux<StepParams<T>, CLOSURE_WEAK>, (unsigned)aux, 128, 0, s, p, a); break;
    case CLOSURE_RHOEQ: e = launch_after_prior(adj::adjoint_aux<StepParams<T>, CLOSURE_RHOEQ>, (unsigned)aux, 128, 0, s, p, a); break;
    case CLOSURE_UNROTATED: e = launch_after_prior(adj::adjoint_aux<StepParams<T>, CLOSURE_UNROTATED>, (unsigned)aux, 128, 0, s, p, a); break;
    default: e = launch_after_prior(adj::adjoint_aux<StepParams<T>, CLOSURE_NONE>, (unsigned)aux, 128, 0, s, p, a); break;
    }
    if (e != cudaSuccess) return -1;
    return launch_after_prior(adj::adjoint_bulk_step<StepParams<T>>, (unsigned)((nodes + 127) / 128), 128, 0, s, p, a) ==
                   cudaSuccess
               ? 0
               : -1;
}

int launch_adjoint_step(const StepParams<double>& p, const adj::AdjArgs& a, cudaStream_t s) { return launch_adjoint(p, a, s); }
int launch_adjoint_step(const StepParams<float>& p, const adj::AdjArgs& a, cudaStream_t s) { return launch_adjoint(p, a, s); }

}  // namespace mrlbm
