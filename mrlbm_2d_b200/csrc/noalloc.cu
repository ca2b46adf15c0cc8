// noalloc.cu -- stepping without any device allocation by the library.
//
// Some hosts own every byte of device memory themselves: a Fortran program whose device
// arrays come from its CUDA Fortran / OpenACC runtime, a framework whose caching allocator
// or arena holds the GPU's memory, a service that freezes allocation after start-up.  Such
// callers cannot let this library call cudaMalloc.  mrlbm_step_noalloc serves them: the
// case comes from a host-only handle (mrlbm_create with device -1 allocates no device
// memory), the caller passes the population buffers, and everything else the step kernel
// needs lives in the fixed-size file-scope arrays below, which every GPU that loads the
// library holds until the process exits.  Nothing here calls cudaMalloc, cudaFree or any
// allocating library routine.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mrlbm.h"
#include "geometry.h"
#include "noalloc.h"
#include "state_io.h"
#include "step_params.h"

namespace mrlbm {

// ---- fixed device storage (the scratch of the step kernel and the case tables) ---------
constexpr int NA_MAX_NB = 1024;                      // curved-wall nodes
constexpr int NA_MAX_BOX = 512 * 512;                // cells of the cylinder bounding box
constexpr int NA_MAX_NY = 8192;                      // rows (the inlet column sum is per row)
constexpr int NA_RING = 4096;                        // stats records buffered per drain
constexpr int NA_MAX_OVR = 64;                       // loaded-state corner overrides

static __device__ __align__(256) double na_geo[G_NFIELDS * NA_MAX_NB];        // FP64 or FP32 tables
static __device__ __align__(256) int na_int[I_NFIELDS * NA_MAX_NB];
static __device__ __align__(256) int na_box[NA_MAX_BOX];
static __device__ __align__(256) double na_partials[2 * NA_MAX_NB + NA_MAX_NY];
static __device__ __align__(256) unsigned na_counter[3];
static __device__ __align__(256) int na_err[1];
static __device__ __align__(256) double na_ring[REC_WORDS * NA_RING];
static __device__ __align__(256) OvrEntry na_ovr[NA_MAX_OVR];

constexpr size_t NA_STATIC_BYTES = sizeof(double) * G_NFIELDS * NA_MAX_NB + sizeof(int) * I_NFIELDS * NA_MAX_NB +
                                   sizeof(int) * NA_MAX_BOX + sizeof(double) * (2 * NA_MAX_NB + NA_MAX_NY) +
                                   sizeof(double) * REC_WORDS * NA_RING + sizeof(OvrEntry) * NA_MAX_OVR + 16;

struct NaSymbols {
    double* geo = nullptr;
    int* ints = nullptr;
    int* box = nullptr;
    double* partials = nullptr;
    unsigned* counter = nullptr;
    int* err = nullptr;
    double* ring = nullptr;
    OvrEntry* ovr = nullptr;
    bool ready = false;
};
constexpr int NA_MAX_DEVICES = 64;
static NaSymbols g_na[NA_MAX_DEVICES];
static std::mutex g_na_mutex;

// Device addresses of the arrays above for the current device.  Host code cannot use the
// array names as device pointers: they are host-side stand-ins.  Looked up once per device
// and cached for the life of the process: the cache assumes the device's primary context
// lives that long (a cudaDeviceReset would leave these addresses stale).
static cudaError_t na_symbols(int dev, NaSymbols** out) {
    if (dev < 0 || dev >= NA_MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_na_mutex);
    NaSymbols& s = g_na[dev];
    if (!s.ready) {
        cudaError_t e;
        if ((e = cudaGetSymbolAddress((void**)&s.geo, na_geo)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void**)&s.ints, na_int)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void**)&s.box, na_box)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void**)&s.partials, na_partials)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void**)&s.counter, na_counter)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void**)&s.err, na_err)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void**)&s.ring, na_ring)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void**)&s.ovr, na_ovr)) != cudaSuccess) return e;
        s.ready = true;
    }
    *out = &s;
    return cudaSuccess;
}

int noalloc_step(NaCase& c, void* d_state, const double* d_f0, int32_t nsteps, double* records, int32_t* n_records,
                 void* stream, std::string& err) {
    if (n_records) *n_records = 0;
    const Geometry& g = *c.geo;
    if (g.nb > NA_MAX_NB) {
        err = "mrlbm_step_noalloc supports at most " + std::to_string(NA_MAX_NB) + " curved-wall nodes (case has " +
              std::to_string(g.nb) + ")";
        return MRLBM_EINVAL;
    }
    if ((int64_t)g.boxmap.size() > NA_MAX_BOX) {
        err = "mrlbm_step_noalloc supports a cylinder bounding box of at most " + std::to_string(NA_MAX_BOX) + " cells";
        return MRLBM_EINVAL;
    }
    if (c.L.ny > NA_MAX_NY) {
        err = "mrlbm_step_noalloc supports at most " + std::to_string(NA_MAX_NY) + " rows";
        return MRLBM_EINVAL;
    }
    if (!d_state) { err = "d_state is NULL"; return MRLBM_EINVAL; }
    // the 128-bit vector shapes read and write d_state with 16-byte accesses; the initial
    // populations are read as doubles
    if ((uintptr_t)d_state % 16 != 0) { err = "d_state must be 16-byte aligned"; return MRLBM_EINVAL; }
    if (d_f0 && (uintptr_t)d_f0 % 8 != 0) { err = "d_f0 must be 8-byte aligned"; return MRLBM_EINVAL; }
    if (d_f0 && c.conflicts.size() > (size_t)NA_MAX_OVR) {
        err = "too many loaded-state overrides (at most " + std::to_string(NA_MAX_OVR) + ")";
        return MRLBM_EINVAL;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    NaSymbols* S = nullptr;
    if (e == cudaSuccess) e = na_symbols(dev, &S);
    if (e != cudaSuccess) { err = std::string("device symbol lookup: ") + cudaGetErrorString(e); return MRLBM_ECUDA; }
    cudaStream_t st = (cudaStream_t)stream;
    const size_t elem = c.precision == MRLBM_FP64 ? 8 : 4;
    const int nb = g.nb;
    // case tables into the fixed arrays (the host copies are the handle's; nothing allocated)
    if (nb > 0) {
        if (c.precision == MRLBM_FP64) {
            e = cudaMemcpyAsync(S->geo, g.tgeo.data(), (size_t)G_NFIELDS * nb * 8, cudaMemcpyHostToDevice, st);
        } else {
            e = cudaMemcpyAsync(S->geo, c.geo32->data(), (size_t)G_NFIELDS * nb * 4, cudaMemcpyHostToDevice, st);
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(S->ints, g.tint.data(), (size_t)I_NFIELDS * nb * sizeof(int), cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess && !g.boxmap.empty())
        e = cudaMemcpyAsync(S->box, g.boxmap.data(), g.boxmap.size() * sizeof(int), cudaMemcpyHostToDevice, st);
    // the arrays keep the previous call's contents: clear what must start at zero
    if (e == cudaSuccess) e = cudaMemsetAsync(S->counter, 0, 3 * sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(S->err, 0, sizeof(int), st);
    if (e != cudaSuccess) { err = std::string("upload: ") + cudaGetErrorString(e); return MRLBM_ECUDA; }
    void* half[2] = {d_state, (char*)d_state + (size_t)c.L.total() * elem};
    bool ovr_live = false;
    int n_ovr = 0;
    if (d_f0) {
        e = launch_scatter_state(c.precision, d_f0, half[0], half[1], c.L, c.xper, c.yper, c.freeslip, c.w, st);
        if (e != cudaSuccess) { err = cudaGetErrorString(e); return MRLBM_ECUDA; }
        n_ovr = (int)c.conflicts.size();                      // checked against NA_MAX_OVR above
        if (n_ovr > 0) {
            e = cudaMemcpyAsync(S->ovr, c.conflicts.data(), (size_t)n_ovr * sizeof(OvrEntry), cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) { err = cudaGetErrorString(e); return MRLBM_ECUDA; }
            e = launch_fill_overrides(c.precision, d_f0, S->ovr, n_ovr, c.L.nx, c.L.ny, c.w, st);
            if (e != cudaSuccess) { err = cudaGetErrorString(e); return MRLBM_ECUDA; }
            ovr_live = true;
        }
        c.cur = 0;
        c.launches += n_ovr > 0 ? 2 : 1;
        if ((e = cudaGetLastError()) != cudaSuccess) { err = cudaGetErrorString(e); return MRLBM_ECUDA; }
    }
    int ring_n = 0, nrec = 0;
    auto drain = [&]() -> int {
        if (ring_n == 0) return MRLBM_OK;
        if (records) {
            cudaError_t e2 = cudaMemcpyAsync(records + (size_t)nrec * REC_WORDS, S->ring,
                                             (size_t)ring_n * REC_WORDS * sizeof(double), cudaMemcpyDeviceToHost, st);
            if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(st);
            if (e2 != cudaSuccess) { err = cudaGetErrorString(e2); return MRLBM_ECUDA; }
        }
        nrec += ring_n;
        ring_n = 0;
        return MRLBM_OK;
    };
    for (int s = 0; s < nsteps; ++s) {
        c.iter += 1;
        const bool stats = c.post_process && c.iter >= c.statsbegin && c.iter <= c.statsend;
        const bool plot = c.plot_enabled && c.iplot > 0 && c.iter % c.iplot == 0;
        int rc;
        if (c.precision == MRLBM_FP64) {
            StepParams<double> p = *c.p64;
            p.src = (const double*)half[c.cur];
            p.dst = (double*)half[1 - c.cur];
            p.bgeo = S->geo;
            p.bint = S->ints;
            p.boxmap = S->box;
            p.partials = S->partials;
            p.counter = S->counter;
            p.errflag = S->err;
            p.rec = stats ? S->ring + (size_t)ring_n * REC_WORDS : nullptr;
            p.do_stats = stats;
            p.zero_solid_u = plot;
            p.iter = c.iter;
            p.macro = nullptr;
            p.u_in = nullptr;
            p.ovr = ovr_live ? S->ovr : nullptr;
            p.n_ovr = ovr_live ? n_ovr : 0;
            rc = launch_step_f64(p, c.tile_cfg, st, 0);
        } else {
            StepParams<float> p = *c.p32;
            p.src = (const float*)half[c.cur];
            p.dst = (float*)half[1 - c.cur];
            p.bgeo = (const float*)S->geo;
            p.bint = S->ints;
            p.boxmap = S->box;
            p.partials = S->partials;
            p.counter = S->counter;
            p.errflag = S->err;
            p.rec = stats ? S->ring + (size_t)ring_n * REC_WORDS : nullptr;
            p.do_stats = stats;
            p.zero_solid_u = plot;
            p.iter = c.iter;
            p.macro = nullptr;
            p.u_in = nullptr;
            p.ovr = ovr_live ? S->ovr : nullptr;
            p.n_ovr = ovr_live ? n_ovr : 0;
            rc = launch_step_f32(p, c.tile_cfg, st, 0);
        }
        c.launches += step_launches(c.precision == MRLBM_FP32, c.tile_cfg);
        if (rc != 0) { err = std::string("kernel launch failed: ") + cudaGetErrorString(cudaGetLastError()); return MRLBM_ECUDA; }
        ovr_live = false;
        c.cur ^= 1;
        if (stats && ++ring_n == NA_RING) {
            int dr = drain();
            if (dr != MRLBM_OK) return dr;
        }
    }
    int dr = drain();
    if (dr != MRLBM_OK) return dr;
    int flag = 0;
    e = cudaMemcpyAsync(&flag, S->err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { err = cudaGetErrorString(e); return MRLBM_ECUDA; }
    if (n_records) *n_records = nrec;
    if (flag) { err = "device flag: NaN or non-positive density"; return MRLBM_EDEVICE_NAN; }
    return MRLBM_OK;
}

size_t noalloc_static_bytes() { return NA_STATIC_BYTES; }

}  // namespace mrlbm
