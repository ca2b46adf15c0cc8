// state_io.h -- conversion between the reference's f(nx,ny,0:8) and the padded pull layout.
#pragma once
#include <cuda_runtime.h>
#include "step_params.h"

namespace mrlbm {

// hl / hr: the lattice is an x-slab whose column 0 / nx+1 holds a neighbour's populations.
// f0 (Fortran order, FP64, device) -> both padded time levels a and b (FP64 values, or FP32
// deviations f - w_k when precision == 32).  Population (i,j,k) goes to the slot its
// next-step gather reads (stream_source).
cudaError_t launch_scatter_state(int precision, const double* f0, void* a, void* b, const Layout& L, int xper,
                                 int yper, int freeslip, const double* w, cudaStream_t s, int hl = 0, int hr = 0);
// padded time level src -> f (Fortran order, FP64, device): the populations the next
// step's gather reads, i.e. the reference's post-streaming f.
cudaError_t launch_gather_state(int precision, const void* src, double* f, const Layout& L, int xper, int yper,
                                int freeslip, const double* w, cudaStream_t s, int hl = 0, int hr = 0);
// override entries (destinations sharing a streaming slot) take their values from f0.
cudaError_t launch_fill_overrides(int precision, const double* f0, OvrEntry* ovr, int n, int nx, int ny,
                                  const double* w, cudaStream_t s);

// Running sums (6 x N: u, v, p, u^2, v^2, p^2) over n steps -> mean (3 x N) and rms of the
// fluctuation sqrt(max(<x^2> - <x>^2, 0)) (3 x N).
cudaError_t launch_field_stats_finalize(const double* sums, double* out, int64_t N, int64_t n, cudaStream_t s);

}  // namespace mrlbm
