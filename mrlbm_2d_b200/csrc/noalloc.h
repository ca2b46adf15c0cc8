// noalloc.h -- host-side interface of noalloc.cu (stepping in caller-owned device memory).
#pragma once
#include <string>
#include <vector>
#include "geometry.h"
#include "step_params.h"

namespace mrlbm {

// Everything mrlbm_step_noalloc needs from a host-only handle.  iter, cur and launches are
// read and updated.
struct NaCase {
    const Geometry* geo = nullptr;
    const std::vector<float>* geo32 = nullptr;   // FP32 copy of geo->tgeo
    int precision = 64;
    Layout L{};
    double w[Q] = {};
    int xper = 0, yper = 0, freeslip = 0;
    int post_process = 0, statsbegin = 0, statsend = 0, iplot = 0;
    bool plot_enabled = false;
    const StepParams<double>* p64 = nullptr;     // common launch parameters, pointers unset
    const StepParams<float>* p32 = nullptr;
    std::vector<OvrEntry> conflicts;             // destinations that share a streaming slot
    int tile_cfg = 1;
    int iter = 0, cur = 0;
    long long launches = 0;
};

int noalloc_step(NaCase& c, void* d_state, const double* d_f0, int32_t nsteps, double* records, int32_t* n_records,
                 void* stream, std::string& err);
size_t noalloc_static_bytes();

}  // namespace mrlbm
