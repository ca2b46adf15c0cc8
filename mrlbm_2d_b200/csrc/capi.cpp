// capi.cpp -- the extern "C" surface of include/mrlbm.h: handle lifetime, device memory,
// state transfer, the time-step loop and the force history ring.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../../include/mrlbm.h"
#include "geometry.h"
#include "adjoint.h"
#include "batch_params.h"
#include "noalloc.h"
#include "state_io.h"
#include "surface.h"
#include "step_params.h"

using namespace mrlbm;

namespace {
thread_local std::string g_create_error;
constexpr int RING_CAP = 8192;                // stats records buffered on the device
constexpr int STREAMS_MAX_STEPS = 1024;       // steps per launch of the per-case streams schedule
}

struct mrlbm_handle {
    mrlbm_config cfg{};
    int precision = MRLBM_FP64;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    Geometry geo;
    Lattice64 lat{};
    double nu = 0, omega = 0;
    int closure = CLOSURE_STRONG;
    Layout L{};
    size_t elem = 8;
    void* buf[2] = {nullptr, nullptr};
    int cur = 0;
    void* d_bgeo = nullptr;
    int* d_bint = nullptr;
    int* d_boxmap = nullptr;
    double* d_partials = nullptr;             // two slots of the per-step record terms
    size_t partials_n = 0;                    // doubles per slot
    int pslot = 0;                            // slot the next stats step writes
    // a stats step whose record sums are deferred to the next launch (StepParams::defer)
    struct Pending { bool on = false; int slot = 0; int rec_idx = 0; int iter = 0; } pend;
    unsigned* d_counter = nullptr;
    double* d_ring = nullptr;
    int ring_n = 0;
    int* d_err = nullptr;
    double* d_macro = nullptr;
    double* d_uin = nullptr;
    bool has_uin = false;
    void* d_body = nullptr;                   // 2 x N body force (T), or null
    bool has_body = false;
    // surface pressure / probe output on statistics steps (2d_mrlbm.f90:462-476, 593-766)
    bool surf_on = false;
    SurfaceTables surf{};
    double *d_quad = nullptr, *d_W = nullptr, *d_sumw = nullptr, *d_sring = nullptr, *d_pring = nullptr;
    int* d_sidx = nullptr;
    int surf_cap = 0, surf_n = 0;
    std::vector<int32_t> surf_iter_dev;       // iterations of the records in the device ring
    std::vector<int32_t> surf_iter;           // drained history
    std::vector<double> surf_hist, probe_hist;
    double* h_ring = nullptr;                 // pinned
    std::vector<double> hist;                 // drained records, REC_WORDS each
    int iter = 0;
    // field statistics (mean/rms of u, v, p) over an iteration window
    double* d_fstat = nullptr;                // 6 x N running sums
    double* d_fstat_out = nullptr;            // 6 x N mean and rms
    int32_t fstat_begin = 0, fstat_end = -1;
    int64_t fstat_n = 0;
    // x-slab of a larger domain (mrlbm_create_slab): global columns gx0 .. gx0 + nx - 1 of gnx
    bool halo_l = false, halo_r = false;
    int gx0 = 1, gnx = 0;
    int tile_cfg = 1;
    long long launches = 0;
    std::string err;
    DevConsts dc{};
    bool host_only = false;
    std::vector<float> geo32;                 // FP32 tables of a host-only FP32 handle
    std::vector<OvrEntry> ovr;                // loaded-state overrides (see OvrEntry)
    bool ovr_live = false;                    // true until the first step after a load
    OvrEntry* d_ovr = nullptr;
    void* adj_ws = nullptr;                   // adjoint workspace, kept between mrlbm_adjoint_drag calls
    size_t adj_ws_bytes = 0;
    double* d_fstage = nullptr;               // f(nx,ny,0:8) staging for state transfers
    // TMA shapes: tensor maps of both time levels, tile-claim counter, persistent CTAs
    unsigned long long* d_tile_ctr = nullptr;
    unsigned long long tile_base = 0;
    int tmap_cfg = -1;
    CUtensorMap tmap[2];
    CUtensorMap tmap_st[2];                   // store maps (box BX x BY) of the TMA-store shapes
    int workers = 0;
    int num_sms = 0;
};

#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            h->err = std::string(#call) + ": " + cudaGetErrorString(e_);                   \
            return MRLBM_ECUDA;                                                            \
        }                                                                                  \
    } while (0)

namespace {

int fail(mrlbm_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

// Streaming-source slot of population (i,j,k) in the padded buffer.
inline int64_t slot_of(const mrlbm_handle* h, int i, int j, int k) {
    const mrlbm_config& c = h->cfg;
    SrcSlot s = stream_source(h->L.nx, h->L.ny, i, j, k, c.x_periodic != 0, c.y_periodic != 0,
                              c.wall_mode == MRLBM_WALL_FREESLIP, h->halo_l, h->halo_r);
    return h->L.at(s.i, s.j, s.k);
}

// Deviation-form constants, computed in FP64 from the reference weights and tables.
// Returns false when a label's Is and Os weight sums differ (the FP32 closure relies on it).
bool make_dev_consts(mrlbm_handle* h) {
    const Lattice64& L = h->lat;
    DevConsts& d = h->dc;
    double sw = 0, cxx = 0, cyy = 0;
    for (int k = 0; k < Q; ++k) { sw += L.w[k]; cxx += L.w[k] * L.hxx[k]; cyy += L.w[k] * L.hyy[k]; }
    d.eps_mass = (float)(sw - 1.0);
    d.cxx = (float)cxx;
    d.cyy = (float)cyy;
    // incoming masks of apply_bc (2d_mrlbm.f90:1254, 1283, 1311, 1339)
    const int masks[4] = {(1 << 0) | (1 << 1) | (1 << 2) | (1 << 4) | (1 << 5) | (1 << 8),
                          (1 << 0) | (1 << 2) | (1 << 3) | (1 << 4) | (1 << 6) | (1 << 7),
                          (1 << 0) | (1 << 1) | (1 << 2) | (1 << 3) | (1 << 5) | (1 << 6),
                          (1 << 0) | (1 << 1) | (1 << 3) | (1 << 4) | (1 << 7) | (1 << 8)};
    double W[4], Sxx[4], Syy[4];
    for (int e = 0; e < 4; ++e) {
        W[e] = 0; Sxx[e] = 0; Syy[e] = 0;
        for (int k = 0; k < Q; ++k)
            if ((masks[e] >> k) & 1) { W[e] += L.w[k]; Sxx[e] += L.w[k] * L.hxx[k]; Syy[e] += L.w[k] * L.hyy[k]; }
    }
    const double om = h->omega;
    d.k_out_mxx = (float)(1.0 + 9.0 * Sxx[0]);
    d.sw_out_yy = (float)Syy[0];
    d.k_in_rho = (float)(4.0 * W[1] + 3.0 * Sxx[1] - 3.0);
    d.k_in_mxx = (float)(1.0 + 9.0 * Sxx[1]);
    d.sw_in_yy = (float)Syy[1];
    d.k_in_rho_inc = (float)(6.0 * W[1] - 5.0);
    for (int e = 0; e < 2; ++e) {
        d.k_w_rho[e] = (float)(12.0 * W[2 + e] - 9.0 - om + 9.0 * (1.0 - om) * Syy[2 + e]);
        d.sw_w_xx[e] = (float)Sxx[2 + e];
        d.k_w_myy[e] = (float)(1.0 + 9.0 * Syy[2 + e]);
        d.k_w_rho_inc[e] = (float)(6.0 * W[2 + e] - 5.0);
        d.w_wall[e] = (float)W[2 + e];
    }
    int incs[16], outs[16];
    link_tables(h->cfg.label15_rule, incs, outs);
    bool ok = true;
    for (int l = 0; l < 16; ++l) {
        double a = 0, b = 0;
        for (int k = 0; k < Q; ++k) {
            if ((incs[l] >> k) & 1) a += L.w[k];
            if ((outs[l] >> k) & 1) b += L.w[k];
        }
        d.lab_w[l] = (float)a;
        if (a != b) ok = false;
    }
    return ok;
}

// Destinations whose streaming slot another destination also uses (the corner populations
// both periodic wraps touch): they keep their own loaded value for the first step.
std::vector<OvrEntry> slot_conflicts(const mrlbm_handle* h) {
    std::vector<std::pair<int64_t, OvrEntry>> cand;
    const int ci[2] = {1, h->L.nx}, cj[2] = {1, h->L.ny};
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int k = 0; k < Q; ++k) cand.push_back({slot_of(h, ci[a], cj[b], k), OvrEntry{ci[a], cj[b], k, 0, 0.0}});
    std::vector<OvrEntry> out;
    for (size_t x = 0; x < cand.size(); ++x)
        for (size_t y = 0; y < cand.size(); ++y)
            if (x != y && cand[x].first == cand[y].first) { out.push_back(cand[x].second); break; }
    return out;
}

// f(nx,ny,0:8) on the host -> both padded time levels: one host->device copy and a scatter
// kernel (state_io.cu).
int upload_state(mrlbm_handle* h, const double* f) {
    const size_t n = (size_t)h->L.nx * h->L.ny * Q;
    if (!h->d_fstage) CK(cudaMalloc((void**)&h->d_fstage, n * sizeof(double)));
    CK(cudaMemcpyAsync(h->d_fstage, f, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    const mrlbm_config& c = h->cfg;
    CK(launch_scatter_state(h->precision, h->d_fstage, h->buf[0], h->buf[1], h->L, c.x_periodic != 0,
                            c.y_periodic != 0, c.wall_mode == MRLBM_WALL_FREESLIP && !c.y_periodic, h->lat.w,
                            h->stream, h->halo_l, h->halo_r));
    ++h->launches;
    h->cur = 0;
    h->ovr = slot_conflicts(h);
    const size_t N = (size_t)h->L.nx * h->L.ny;
    for (OvrEntry& e : h->ovr) {
        const double v = f[(size_t)(e.i - 1) + (size_t)h->L.nx * (e.j - 1) + N * e.k];
        e.v = h->precision == MRLBM_FP64 ? v : (double)(float)(v - h->lat.w[e.k]);
    }
    if (!h->ovr.empty()) {                // at most the 4 x 9 corner slots; allocated once
        if (!h->d_ovr) CK(cudaMalloc((void**)&h->d_ovr, 4 * Q * sizeof(OvrEntry)));
        CK(cudaMemcpyAsync(h->d_ovr, h->ovr.data(), h->ovr.size() * sizeof(OvrEntry), cudaMemcpyHostToDevice,
                           h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    h->ovr_live = !h->ovr.empty();
    return MRLBM_OK;
}

// Sum the terms of a stats step whose record was deferred (one small launch on the handle's
// stream) so the device ring holds every record of the steps launched so far.
int finish_pending(mrlbm_handle* h) {
    if (!h->pend.on) return MRLBM_OK;
    h->pend.on = false;
    if (launch_finish_record(h->d_partials + (size_t)h->pend.slot * h->partials_n, h->geo.nb, h->L.ny, h->halo_l ? 1 : 0,
                             h->d_ring + (size_t)h->pend.rec_idx * REC_WORDS, h->pend.iter, h->stream) != 0)
        return fail(h, MRLBM_ECUDA, "record sums launch failed");
    ++h->launches;
    return MRLBM_OK;
}

int drain_ring(mrlbm_handle* h) {
    int prc = finish_pending(h);
    if (prc != MRLBM_OK) return prc;
    if (h->ring_n == 0) return MRLBM_OK;
    CK(cudaMemcpyAsync(h->h_ring, h->d_ring, (size_t)h->ring_n * REC_WORDS * sizeof(double),
                       cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->hist.insert(h->hist.end(), h->h_ring, h->h_ring + (size_t)h->ring_n * REC_WORDS);
    h->ring_n = 0;
    return MRLBM_OK;
}

template <class T>
void fill_common(mrlbm_handle* h, StepParams<T>& p) {
    const mrlbm_config& c = h->cfg;
    p.L = h->L;
    for (int k = 0; k < Q; ++k) p.w[k] = (T)h->lat.w[k];
    p.hm = (T)h->lat.hm;
    p.hp = (T)h->lat.hp;
    p.omega = (T)h->omega;
    p.omega1 = (T)(1.0 - h->omega);
    p.uinlet = (T)c.uo;
    p.vinlet = (T)0.0;
    p.u_in = nullptr;
    p.xper = c.x_periodic != 0;
    p.yper = c.y_periodic != 0;
    p.freeslip = c.wall_mode == MRLBM_WALL_FREESLIP && !c.y_periodic;
    p.walls_ref = c.wall_mode == MRLBM_WALL_REFERENCE && !c.y_periodic;
    p.incomp_bc = c.incomp_bc != 0;
    p.incomp_bulk = c.incomp_bulk != 0;
    p.nb = h->geo.nb;
    p.bint = h->d_bint;
    p.bgeo = (const T*)h->d_bgeo;
    p.closure = h->closure;
    p.vel_interp = c.vel_interp != 0;
    p.mom_interp = c.mom_interp != 0;
    p.box_x0 = h->geo.box_x0;
    p.box_y0 = h->geo.box_y0;
    p.box_w = h->geo.box_w;
    p.box_h = h->geo.box_h;
    p.boxmap = h->d_boxmap;
    p.label15_allnine = c.label15_rule == MRLBM_LABEL15_ALLNINE;
    p.partials = h->d_partials;
    p.counter = h->d_counter;
    p.halo_l = h->halo_l;
    p.halo_r = h->halo_r;
    p.node_force = nullptr;
    p.errflag = h->d_err;
    p.dc = h->dc;
}

// Claims one TMA step makes on the tile counter (see step_tma.cuh): every tile once plus
// STAGES failing claims per persistent CTA.
unsigned long long tma_claims_host(int nx, int ny, int bx, int by, int stages, int workers) {
    return (unsigned long long)(((nx + bx - 1) / bx) * ((ny + by - 1) / by)) +
           (unsigned long long)workers * (unsigned long long)stages;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* ptr = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)ptr;
    }
    return fn;
}

// Tensor maps (one per time level) and persistent CTA count for a TMA shape.  The map views a
// level as a 2-D array of pitch columns and 9*(ny+2) rows (the nine direction planes stacked).
int prepare_tma(mrlbm_handle* h, int cfg) {
    if (h->tmap_cfg == cfg) return MRLBM_OK;
    auto enc = tensor_map_encoder();
    if (!enc) return fail(h, MRLBM_EUNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
    int bw, bh, st;
    tma_box(h->precision, cfg, &bw, &bh, &st);
    const int per_sm = tma_ctas_per_sm(h->precision, cfg);
    if (per_sm < 0) {
        cudaGetLastError();
        return fail(h, MRLBM_ECUDA, std::string("TMA occupancy query: ") + cudaGetErrorString((cudaError_t)-per_sm));
    }
    if (per_sm == 0) return fail(h, MRLBM_EUNSUPPORTED, "TMA shape does not fit this precision");
    if (!h->d_tile_ctr) {
        CK(cudaMalloc((void**)&h->d_tile_ctr, sizeof(unsigned long long)));
        CK(cudaMemsetAsync(h->d_tile_ctr, 0, sizeof(unsigned long long), h->stream));
        h->tile_base = 0;
    }
    for (int b = 0; b < 2; ++b) {
        cuuint64_t dims[2] = {(cuuint64_t)h->L.pitch, (cuuint64_t)Q * (h->L.ny + 2)};
        cuuint64_t strides[1] = {(cuuint64_t)h->L.pitch * h->elem};
        cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
        cuuint32_t estr[2] = {1, 1};
        CUresult r = enc(&h->tmap[b], h->elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                         2, h->buf[b], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return fail(h, MRLBM_EUNSUPPORTED, "tensor map encoding failed");
        if (is_tma_store_cfg(cfg)) {
            cuuint32_t sbox[2] = {(cuuint32_t)tma_cfg(cfg).bx, (cuuint32_t)bh};
            r = enc(&h->tmap_st[b], h->elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                    h->buf[b], dims, strides, sbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return fail(h, MRLBM_EUNSUPPORTED, "store tensor map encoding failed");
        }
    }
    h->workers = h->num_sms * per_sm;
    h->tmap_cfg = cfg;
    return MRLBM_OK;
}

// Surface pressure and probes of the step just launched (its input level is buf[cur]).
int drain_surface(mrlbm_handle* h) {
    if (h->surf_n == 0) return MRLBM_OK;
    const int nb = h->geo.nb;
    const size_t a = h->surf_hist.size(), b = h->probe_hist.size();
    h->surf_hist.resize(a + (size_t)h->surf_n * 2 * nb);
    h->probe_hist.resize(b + (size_t)h->surf_n * 12);
    CK(cudaMemcpyAsync(h->surf_hist.data() + a, h->d_sring, (size_t)h->surf_n * 2 * nb * sizeof(double),
                       cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(h->probe_hist.data() + b, h->d_pring, (size_t)h->surf_n * 12 * sizeof(double),
                       cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->surf_iter.insert(h->surf_iter.end(), h->surf_iter_dev.begin(), h->surf_iter_dev.end());
    h->surf_iter_dev.clear();
    h->surf_n = 0;
    return MRLBM_OK;
}

int surface_step(mrlbm_handle* h) {
    if (h->surf_n == h->surf_cap) {
        int rc = drain_surface(h);
        if (rc != MRLBM_OK) return rc;
    }
    const int nb = h->geo.nb;
    double* rec = h->d_sring + (size_t)h->surf_n * 2 * nb;
    double* prec = h->d_pring + (size_t)h->surf_n * 12;
    int rc;
    if (h->precision == MRLBM_FP64) {
        StepParams<double> p{};
        fill_common(h, p);
        p.src = (const double*)h->buf[h->cur];
        rc = launch_surface_f64(p, h->surf, rec, prec, h->stream);
    } else {
        StepParams<float> p{};
        fill_common(h, p);
        p.src = (const float*)h->buf[h->cur];
        rc = launch_surface_f32(p, h->surf, rec, prec, h->stream);
    }
    h->launches += 2;
    if (rc != 0) return fail(h, MRLBM_ECUDA, "surface kernel launch failed");
    h->surf_iter_dev.push_back(h->iter);
    ++h->surf_n;
    return MRLBM_OK;
}

// Deferred record sums for a step launched through launch_one: this step's terms go to the
// slot pslot, and the pending step's terms (the other slot) are summed by this launch.
template <class T>
void set_deferred(const mrlbm_handle* h, StepParams<T>& p) {
    p.defer = 1;
    p.partials = h->d_partials + (size_t)h->pslot * h->partials_n;
    if (h->pend.on) {
        p.prev_partials = h->d_partials + (size_t)h->pend.slot * h->partials_n;
        p.prev_rec = h->d_ring + (size_t)h->pend.rec_idx * REC_WORDS;
        p.prev_iter = h->pend.iter;
    }
}

int launch_one(mrlbm_handle* h, bool stats, bool plot, bool macro) {
    const int tc = h->tile_cfg;
    const bool fstat = h->d_fstat && h->iter >= h->fstat_begin && h->iter <= h->fstat_end;
    const bool tma = is_tma_cfg(tc);
    if (tma) {
        int prc = prepare_tma(h, tc);
        if (prc != MRLBM_OK) return prc;
    }
    int rc;
    if (h->precision == MRLBM_FP64) {
        StepParams<double> p{};
        fill_common(h, p);
        set_deferred(h, p);
        p.src = (const double*)h->buf[h->cur];
        p.dst = (double*)h->buf[1 - h->cur];
        p.u_in = h->has_uin ? h->d_uin : nullptr;
        p.body = h->has_body ? (const double*)h->d_body : nullptr;
        p.ovr = h->ovr_live ? h->d_ovr : nullptr;
        p.n_ovr = h->ovr_live ? (int)h->ovr.size() : 0;
        p.zero_solid_u = plot;
        p.do_stats = stats;
        p.rec = stats ? h->d_ring + (size_t)h->ring_n * REC_WORDS : nullptr;
        p.iter = h->iter;
        p.macro = macro ? h->d_macro : nullptr;
        p.fstat = fstat ? h->d_fstat : nullptr;
        if (tma) {
            p.tmap = h->tmap[h->cur];
            p.tmap_st = h->tmap_st[1 - h->cur];
            p.tile_ctr = h->d_tile_ctr;
            p.tile_base = h->tile_base;
        }
        rc = launch_step_f64(p, tc, h->stream, h->workers);
    } else {
        StepParams<float> p{};
        fill_common(h, p);
        set_deferred(h, p);
        p.src = (const float*)h->buf[h->cur];
        p.dst = (float*)h->buf[1 - h->cur];
        p.u_in = h->has_uin ? (const float*)h->d_uin : nullptr;
        p.body = h->has_body ? (const float*)h->d_body : nullptr;
        p.ovr = h->ovr_live ? h->d_ovr : nullptr;
        p.n_ovr = h->ovr_live ? (int)h->ovr.size() : 0;
        p.zero_solid_u = plot;
        p.do_stats = stats;
        p.rec = stats ? h->d_ring + (size_t)h->ring_n * REC_WORDS : nullptr;
        p.iter = h->iter;
        p.macro = macro ? h->d_macro : nullptr;
        p.fstat = fstat ? h->d_fstat : nullptr;
        if (tma) {
            p.tmap = h->tmap[h->cur];
            p.tmap_st = h->tmap_st[1 - h->cur];
            p.tile_ctr = h->d_tile_ctr;
            p.tile_base = h->tile_base;
        }
        rc = launch_step_f32(p, tc, h->stream, h->workers);
    }
    const int nl = step_launches(h->precision == MRLBM_FP32, tc);
    h->launches += nl;
    if (rc == -2) {
        h->launches -= nl;
        return fail(h, MRLBM_EUNSUPPORTED, "tile shape does not fit this precision");
    }
    if (rc != 0) {
        h->err = std::string("kernel launch failed: ") + cudaGetErrorString(cudaGetLastError());
        return MRLBM_ECUDA;
    }
    // the pending record (if any) is summed by this launch; this step's, if a stats step, is next
    h->pend.on = false;
    if (stats) {
        h->pend = mrlbm_handle::Pending{true, h->pslot, h->ring_n, h->iter};
        h->pslot ^= 1;
    }
    if (tma) {
        int bw, bh, st;
        tma_box(h->precision, tc, &bw, &bh, &st);
        h->tile_base += tma_claims_host(h->L.nx, h->L.ny, tma_cfg(tc).bx, bh, st, h->workers);
    }
    if (stats && h->surf_on) {
        int src = surface_step(h);
        if (src != MRLBM_OK) return src;
    }
    h->cur ^= 1;
    h->ovr_live = false;
    if (stats) ++h->ring_n;
    if (fstat) ++h->fstat_n;
    return MRLBM_OK;
}

void free_all(mrlbm_handle* h) {
    if (h->host_only) return;
    cudaSetDevice(h->device);
    for (void* p : {h->buf[0], h->buf[1], h->d_bgeo, (void*)h->d_bint, (void*)h->d_boxmap, (void*)h->d_partials,
                    (void*)h->d_counter, (void*)h->d_ring, (void*)h->d_err, (void*)h->d_macro, (void*)h->d_uin, h->d_body, (void*)h->d_ovr, h->adj_ws, (void*)h->d_fstage,
                    (void*)h->d_tile_ctr, (void*)h->d_fstat, (void*)h->d_fstat_out, (void*)h->d_quad, (void*)h->d_W,
                    (void*)h->d_sumw, (void*)h->d_sring, (void*)h->d_pring, (void*)h->d_sidx})
        if (p) cudaFree(p);
    if (h->h_ring) cudaFreeHost(h->h_ring);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
}

// Geometry of the x-slab gx0..gx1 of a built domain: node classes sliced, wall-node and
// stencil column indices shifted; the wall-point coordinates, centre and angles stay global
// so every derived value keeps its bits.  The cylinder with its bilinear stencils must lie
// strictly inside one slab (or the slab holds none of it).
int slice_geometry(const Geometry& g, int gx0, int gx1, Geometry& s, std::string& err) {
    const int nxl = gx1 - gx0 + 1, ny = g.ny, sh = gx0 - 1;
    s = g;
    s.nx = nxl;
    s.cls.assign((size_t)nxl * ny, 0);
    bool any = false;
    for (int j = 1; j <= ny; ++j)
        for (int i = gx0; i <= gx1; ++i) {
            const int8_t c = g.cls[(size_t)(i - 1) + (size_t)g.nx * (j - 1)];
            s.cls[(size_t)(i - gx0) + (size_t)nxl * (j - 1)] = c;
            any = any || c != 0;
        }
    if (!g.cylinder || g.nb == 0 || !any) {
        // no part of the cylinder here: a plain channel slab (any cylinder node outside it)
        for (int j = 1; j <= ny && g.cylinder; ++j)
            for (int i = gx0 - 1; i <= gx1 + 1; ++i)
                if (i >= 1 && i <= g.nx && g.cls[(size_t)(i - 1) + (size_t)g.nx * (j - 1)] != 0) {
                    err = "the cylinder touches the slab's halo columns";
                    return MRLBM_EGEOMETRY;
                }
        s.nb = 0;
        s.bi.clear(); s.bj.clear(); s.label.clear(); s.delta.clear(); s.ref.clear(); s.sten.clear(); s.theta.clear();
        s.tint.clear(); s.tgeo.clear(); s.boxmap.clear();
        s.box_x0 = 1; s.box_y0 = 1; s.box_w = 0; s.box_h = 0;
        s.cylinder = false;
        return MRLBM_OK;
    }
    // every wall node, solid node and stencil node strictly inside the slab
    auto inside = [&](int i) { return i > gx0 && i < gx1; };
    if (!inside(g.box_x0) || !inside(g.box_x0 + g.box_w - 1)) {
        err = "the cylinder is cut by a slab boundary";
        return MRLBM_EGEOMETRY;
    }
    for (int l = 0; l < g.nb; ++l) {
        for (int m = 0; m < 12; ++m)
            if (!inside(g.sten[24 * (size_t)l + 8 * (m / 4) + (m % 4)])) {
                err = "a bilinear stencil of the cylinder crosses a slab boundary";
                return MRLBM_EGEOMETRY;
            }
        s.bi[l] = g.bi[l] - sh;
        for (int m = 0; m < 12; ++m) s.sten[24 * (size_t)l + 8 * (m / 4) + (m % 4)] -= sh;
        s.tint[(size_t)I_NODEI * g.nb + l] -= sh;
        for (int m = 0; m < 12; ++m) s.tint[(size_t)(I_SI + m) * g.nb + l] -= sh;
    }
    s.box_x0 = g.box_x0 - sh;
    return MRLBM_OK;
}

}  // namespace

extern "C" {

size_t mrlbm_config_sizeof(void) { return sizeof(mrlbm_config); }

int mrlbm_config_defaults(mrlbm_config* cfg) {
    if (!cfg) return MRLBM_EINVAL;
    config_defaults(*cfg);
    return MRLBM_OK;
}

int mrlbm_config_from_namelist(const char* path, mrlbm_config* cfg) {
    if (!path || !cfg) return MRLBM_EINVAL;
    std::string err;
    int rc = read_namelist_file(path, *cfg, err);
    if (rc != MRLBM_OK) g_create_error = "Error while reading input.dat file... (" + err + ")";
    return rc;
}

int mrlbm_config_resolve_geometry(mrlbm_config* cfg) {
    if (!cfg) return MRLBM_EINVAL;
    if (cfg->geometry_mode != MRLBM_GEOM_REFERENCE || !cfg->channel_with_cylinder) return MRLBM_OK;
    int nx, ny;
    double x, y, r;
    resolve_domain(*cfg, nx, ny, x, y, r);
    cfg->nx = nx; cfg->ny = ny; cfg->x_c = x; cfg->y_c = y; cfg->r_c = r;
    return MRLBM_OK;
}

static int create_impl(const mrlbm_config* cfg, int precision, int device, int sx0, int sx1, mrlbm_handle** out) {
    if (!cfg || !out) return MRLBM_EINVAL;
    *out = nullptr;
    if (precision != MRLBM_FP64 && precision != MRLBM_FP32) {
        g_create_error = "precision must be 64 or 32";
        return MRLBM_EINVAL;
    }
    mrlbm_handle* h = new mrlbm_handle();
    h->cfg = *cfg;
    h->precision = precision;
    h->device = device;
    h->elem = precision == MRLBM_FP64 ? 8 : 4;
    const mrlbm_config& c = h->cfg;
    auto bail = [&](int code, const std::string& m) {
        g_create_error = m;
        free_all(h);
        delete h;
        return code;
    };
    if (c.Re <= 0 || !(c.uo == c.uo)) return bail(MRLBM_EINVAL, "Re must be positive");
    if (c.channel_with_cylinder && c.rotated_coordinate && (c.strong_mass_bc || c.eq_mass_bc || c.weak_mass_bc) &&
        !c.mom_interp)
        return bail(MRLBM_EUNSUPPORTED,
                    "rotated closures read mxxp/myyp, which the reference sets only when mom_interp is true");
    int nx, ny;
    double xc, yc, rc;
    resolve_domain(c, nx, ny, xc, yc, rc);
    if (nx < 4 || ny < 4) return bail(MRLBM_EINVAL, "nx and ny must be >= 4");
    h->cfg.nx = nx; h->cfg.ny = ny; h->cfg.x_c = xc; h->cfg.y_c = yc; h->cfg.r_c = rc;
    std::string err;
    int grc = build_geometry(c, nx, ny, xc, yc, rc, h->geo, err);
    if (grc != MRLBM_OK) return bail(grc, err);
    h->gnx = nx;
    const int gnx = nx;
    if (sx0 > 0) {                                   // one x-slab of the domain
        if (c.x_periodic) return bail(MRLBM_EUNSUPPORTED, "x-slabs of an x-periodic domain");
        if (sx0 < 1 || sx1 > nx || sx1 - sx0 + 1 < 4) return bail(MRLBM_EINVAL, "slab columns out of range");
        Geometry full = h->geo;
        grc = slice_geometry(full, sx0, sx1, h->geo, err);
        if (grc != MRLBM_OK) return bail(grc, err);
        h->gx0 = sx0;
        h->halo_l = sx0 > 1;
        h->halo_r = sx1 < nx;
        nx = sx1 - sx0 + 1;
    }
    h->lat = make_lattice();
    // viscosity and relaxation, 2d_mrlbm.f90:133-135
    h->nu = c.uo * (double)(ny - 1) / c.Re;
    if (c.channel_with_cylinder) {
        const double Lr = c.nu_length == MRLBM_NU_DIAMETER ? rc : h->geo.r_cyl;
        h->nu = c.uo * (2.0 * Lr) / c.Re;
    }
    h->omega = 1.0 / ((3.0 * h->nu) + (1.0 / 2.0));
    // curved-wall variant actually applied (2d_mrlbm.f90:280-311): the last flag called wins
    if (!c.rotated_coordinate) h->closure = CLOSURE_UNROTATED;
    else if (c.weak_mass_bc) h->closure = CLOSURE_WEAK;
    else if (c.eq_mass_bc) h->closure = CLOSURE_RHOEQ;
    else if (c.strong_mass_bc) h->closure = CLOSURE_STRONG;
    else h->closure = CLOSURE_NONE;
    if (!make_dev_consts(h) && precision == MRLBM_FP32)
        return bail(MRLBM_EUNSUPPORTED, "FP32 closure needs equal Is/Os weight sums for every label");

    h->L = make_layout(nx, ny, precision == MRLBM_FP64 ? 16 : 32);
    if (h->L.total() >= (int64_t)1 << 31) return bail(MRLBM_EINVAL, "grid too large for one handle (2^31 populations)");
    const char* tc = std::getenv("MRLBM_TILE_CFG");
    if (tc) h->tile_cfg = std::max(0, std::min(N_ALL_CFGS - 1, std::atoi(tc)));
    if (device == -1) {            // host-only handle: configuration and geometry, no device state
        h->host_only = true;
        h->iter = 1;
        if (precision == MRLBM_FP32) h->geo32.assign(h->geo.tgeo.begin(), h->geo.tgeo.end());
        *out = h;
        return MRLBM_OK;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return bail(MRLBM_ENODEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return bail(MRLBM_EINVAL, "device index out of range");
    auto ck = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess) { g_create_error = std::string(what) + ": " + cudaGetErrorString(e); return false; }
        return true;
    };
    bool ok = ck(cudaSetDevice(device), "cudaSetDevice") &&
              ck(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device), "SM count") &&
              ck(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    h->stream = h->own_stream;
    const size_t bytes = (size_t)h->L.total() * h->elem;
    ok = ok && ck(cudaMalloc(&h->buf[0], bytes), "cudaMalloc state") && ck(cudaMalloc(&h->buf[1], bytes), "cudaMalloc state");
    const int nb = h->geo.nb;
    const size_t ngeo = (size_t)G_NFIELDS * std::max(nb, 1), nint = (size_t)I_NFIELDS * std::max(nb, 1);
    ok = ok && ck(cudaMalloc(&h->d_bgeo, ngeo * h->elem), "cudaMalloc tables") &&
         ck(cudaMalloc((void**)&h->d_bint, nint * sizeof(int)), "cudaMalloc tables");
    const size_t nbox = std::max<size_t>(h->geo.boxmap.size(), 1);
    ok = ok && ck(cudaMalloc((void**)&h->d_boxmap, nbox * sizeof(int)), "cudaMalloc boxmap");
    const size_t nscratch = 2 * (size_t)nb + (size_t)ny + 8;
    h->partials_n = nscratch;
    ok = ok && ck(cudaMalloc((void**)&h->d_partials, 2 * nscratch * sizeof(double)), "cudaMalloc partials") &&
         ck(cudaMalloc((void**)&h->d_counter, 3 * sizeof(unsigned)), "cudaMalloc counter") &&
         ck(cudaMalloc((void**)&h->d_ring, (size_t)RING_CAP * REC_WORDS * sizeof(double)), "cudaMalloc ring") &&
         ck(cudaMalloc((void**)&h->d_err, sizeof(int)), "cudaMalloc err") &&
         ck(cudaMallocHost((void**)&h->h_ring, (size_t)RING_CAP * REC_WORDS * sizeof(double)), "cudaMallocHost ring");
    if (!ok) { std::string m = g_create_error; return bail(MRLBM_ECUDA, m); }
    if (nb > 0) {
        if (precision == MRLBM_FP64) {
            ok = ck(cudaMemcpy(h->d_bgeo, h->geo.tgeo.data(), ngeo * 8, cudaMemcpyHostToDevice), "upload tables");
        } else {
            std::vector<float> t(h->geo.tgeo.begin(), h->geo.tgeo.end());
            ok = ck(cudaMemcpy(h->d_bgeo, t.data(), ngeo * 4, cudaMemcpyHostToDevice), "upload tables");
        }
        ok = ok && ck(cudaMemcpy(h->d_bint, h->geo.tint.data(), nint * sizeof(int), cudaMemcpyHostToDevice), "upload tables");
    }
    if (!h->geo.boxmap.empty())
        ok = ok && ck(cudaMemcpy(h->d_boxmap, h->geo.boxmap.data(), h->geo.boxmap.size() * sizeof(int),
                                 cudaMemcpyHostToDevice), "upload boxmap");
    ok = ok && ck(cudaMemset(h->d_counter, 0, 3 * sizeof(unsigned)), "memset") && ck(cudaMemset(h->d_err, 0, sizeof(int)), "memset");
    if (!ok) { std::string m = g_create_error; return bail(MRLBM_ECUDA, m); }
    std::vector<double> f0;
    initial_state(h->cfg, h->lat, gnx, ny, f0);
    if (nx != gnx) {                                 // the slab's columns of the domain's start
        std::vector<double> fs((size_t)nx * ny * Q);
        for (int k = 0; k < Q; ++k)
            for (int j = 1; j <= ny; ++j)
                std::memcpy(&fs[(size_t)nx * ny * k + (size_t)nx * (j - 1)],
                            &f0[(size_t)gnx * ny * k + (size_t)gnx * (j - 1) + (h->gx0 - 1)], nx * sizeof(double));
        f0.swap(fs);
    }
    int urc = upload_state(h, f0.data());
    if (urc != MRLBM_OK) { std::string m = h->err; return bail(urc, m); }
    // the main loop runs iter = restart_step+1, ... with restart_step initialised to 1
    // (2d_mrlbm.f90:7, 229): a fresh run's first step is iter 2
    h->iter = 1;
    *out = h;
    return MRLBM_OK;
}

int mrlbm_create(const mrlbm_config* cfg, int precision, int device, mrlbm_handle** out) {
    return create_impl(cfg, precision, device, 0, 0, out);
}

int mrlbm_create_slab(const mrlbm_config* cfg, int precision, int device, int32_t gx0, int32_t gx1,
                      mrlbm_handle** out) {
    if (gx0 < 1) return MRLBM_EINVAL;
    return create_impl(cfg, precision, device, gx0, gx1, out);
}

// Halo columns: side 0 is the left face (the populations moving left, k = 3, 6, 7, of column 1
// go out; the left neighbour's k = 1, 5, 8 come into column 0), side 1 the right face (k = 1,
// 5, 8 of column nx out; k = 3, 6, 7 into column nx + 1).  3 x ny values of the handle's
// storage type per face, k-major, rows 1..ny.
static const int HALO_OUT[2][3] = {{3, 6, 7}, {1, 5, 8}};
static const int HALO_IN[2][3] = {{1, 5, 8}, {3, 6, 7}};

int mrlbm_halo_size(const mrlbm_handle* h, int64_t* n_values, int32_t* elem_bytes) {
    if (!h || !n_values) return MRLBM_EINVAL;
    *n_values = 3 * (int64_t)h->L.ny;
    if (elem_bytes) *elem_bytes = h->elem;
    return MRLBM_OK;
}

// One halo face between a slab's time level (next = false: the current state, true: the
// level the next step writes) and a flat device buffer, or straight into a neighbour's
// buffer peer_dst (same time level) on the handle's stream (or on `on`, if given).
static int halo_copy(mrlbm_handle* h, int side, void* dev, bool pack, void* peer_dst, const mrlbm_handle* peer,
                     bool next = false, cudaStream_t on = nullptr) {
    if (!h || side < 0 || side > 1) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    CK(cudaSetDevice(h->device));
    const int ny = h->L.ny;
    const size_t e = h->elem, pitch_b = (size_t)h->L.pitch * e;
    char* base = (char*)h->buf[next ? 1 - h->cur : h->cur];
    cudaStream_t st = on ? on : h->stream;
    for (int q = 0; q < 3; ++q) {
        if (pack) {
            const int i = side == 0 ? 1 : h->L.nx, k = HALO_OUT[side][q];
            const char* src = base + (size_t)h->L.at(i, 1, k) * e;
            if (peer) {                              // straight into the neighbour's ghost column
                const int pi = side == 0 ? peer->L.nx + 1 : 0;
                char* dst = (char*)peer_dst + (size_t)peer->L.at(pi, 1, k) * e;
                CK(cudaMemcpy2DAsync(dst, (size_t)peer->L.pitch * e, src, pitch_b, e, ny, cudaMemcpyDefault, st));
            } else {
                CK(cudaMemcpy2DAsync((char*)dev + (size_t)q * ny * e, e, src, pitch_b, e, ny, cudaMemcpyDefault, st));
            }
        } else {
            const int i = side == 0 ? 0 : h->L.nx + 1, k = HALO_IN[side][q];
            char* dst = base + (size_t)h->L.at(i, 1, k) * e;
            CK(cudaMemcpy2DAsync(dst, pitch_b, (const char*)dev + (size_t)q * ny * e, e, e, ny, cudaMemcpyDefault, st));
        }
    }
    return MRLBM_OK;
}

int mrlbm_halo_pack(mrlbm_handle* h, int32_t side, void* dst) {
    if (!dst) return MRLBM_EINVAL;
    return halo_copy(h, side, dst, true, nullptr, nullptr);
}

int mrlbm_halo_unpack(mrlbm_handle* h, int32_t side, const void* src) {
    if (!src) return MRLBM_EINVAL;
    return halo_copy(h, side, const_cast<void*>(src), false, nullptr, nullptr);
}

int mrlbm_halo_pack_next(mrlbm_handle* h, int32_t side, void* dst) {
    if (!dst) return MRLBM_EINVAL;
    return halo_copy(h, side, dst, true, nullptr, nullptr, true);
}

int mrlbm_halo_unpack_next(mrlbm_handle* h, int32_t side, const void* src) {
    if (!src) return MRLBM_EINVAL;
    return halo_copy(h, side, const_cast<void*>(src), false, nullptr, nullptr, true);
}

// Halo-face columns of the next step into the next time level (face_kernel), with the
// parameters the step will use, minus its statistics, field sums and macroscopic output.
int mrlbm_step_faces(mrlbm_handle* h) {
    if (!h) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    if (!h->halo_l && !h->halo_r) return MRLBM_OK;
    CK(cudaSetDevice(h->device));
    const mrlbm_config& c = h->cfg;
    const int iter = h->iter + 1;
    const bool plot = c.post_process && c.iplot > 0 && iter % c.iplot == 0 && (c.channel_with_cylinder || c.channel_with_square);
    // the kernel instantiation the step will use when it asks for no macroscopic output
    const bool full = h->has_body || (h->d_fstat && iter >= h->fstat_begin && iter <= h->fstat_end);
    int rc;
    if (h->precision == MRLBM_FP64) {
        StepParams<double> p{};
        fill_common(h, p);
        p.src = (const double*)h->buf[h->cur];
        p.dst = (double*)h->buf[1 - h->cur];
        p.u_in = h->has_uin ? h->d_uin : nullptr;
        p.body = h->has_body ? (const double*)h->d_body : nullptr;
        p.ovr = h->ovr_live ? h->d_ovr : nullptr;
        p.n_ovr = h->ovr_live ? (int)h->ovr.size() : 0;
        p.zero_solid_u = plot;
        p.iter = iter;
        rc = launch_face_f64(p, full, h->stream);
    } else {
        StepParams<float> p{};
        fill_common(h, p);
        p.src = (const float*)h->buf[h->cur];
        p.dst = (float*)h->buf[1 - h->cur];
        p.u_in = h->has_uin ? (const float*)h->d_uin : nullptr;
        p.body = h->has_body ? (const float*)h->d_body : nullptr;
        p.ovr = h->ovr_live ? h->d_ovr : nullptr;
        p.n_ovr = h->ovr_live ? (int)h->ovr.size() : 0;
        p.zero_solid_u = plot;
        p.iter = iter;
        rc = launch_face_f32(p, full, h->stream);
    }
    ++h->launches;
    if (rc != 0) return fail(h, MRLBM_ECUDA, std::string("face kernel launch failed: ") + cudaGetErrorString(cudaGetLastError()));
    return MRLBM_OK;
}

int mrlbm_slabs_step(mrlbm_handle** hs, int32_t n, int32_t nsteps) {
    if (!hs || n < 1 || nsteps < 0) return MRLBM_EINVAL;
    for (int s = 0; s < n; ++s) {
        if (!hs[s] || hs[s]->host_only || hs[s]->precision != hs[0]->precision || hs[s]->L.ny != hs[0]->L.ny)
            return MRLBM_EINVAL;
        if (s > 0 && (!hs[s]->halo_l || !hs[s - 1]->halo_r || hs[s]->gx0 != hs[s - 1]->gx0 + hs[s - 1]->L.nx))
            return fail(hs[s], MRLBM_EINVAL, "slabs must be given left to right, adjacent");
    }
    // Per step and slab: the face kernel writes the halo-face columns of the next level
    // (event face), the step kernel then computes the whole slab on the slab's stream while a
    // side stream copies the faces into the neighbours' next levels.  A copy into a neighbour's
    // level waits for the neighbour's previous step, which read that level; a slab's next face
    // kernel waits for the copies into its level.
    std::vector<cudaEvent_t> face(n), done(n), halo(n);
    std::vector<cudaStream_t> side(n, nullptr);
    int rc = MRLBM_OK;
    for (int s = 0; s < n && rc == MRLBM_OK; ++s) {
        if (cudaSetDevice(hs[s]->device) != cudaSuccess ||
            cudaStreamCreateWithFlags(&side[s], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&face[s], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&done[s], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&halo[s], cudaEventDisableTiming) != cudaSuccess)
            rc = fail(hs[s], MRLBM_ECUDA, "stream or event creation");
        else {
            cudaEventRecord(done[s], hs[s]->stream);         // "previous step" of the first step
            cudaEventRecord(halo[s], hs[s]->stream);
        }
    }
    for (int t = 0; t < nsteps && rc == MRLBM_OK; ++t) {
        for (int s = 0; s < n; ++s) {                          // copies of step t wait for the
            cudaSetDevice(hs[s]->device);                      // neighbours' step t-1
            if (s > 0) cudaStreamWaitEvent(side[s], done[s - 1], 0);
            if (s + 1 < n) cudaStreamWaitEvent(side[s], done[s + 1], 0);
        }
        for (int s = 0; s < n && rc == MRLBM_OK; ++s) {
            cudaSetDevice(hs[s]->device);
            if (s > 0) cudaStreamWaitEvent(hs[s]->stream, halo[s - 1], 0);      // right-going halo of t-1
            if (s + 1 < n) cudaStreamWaitEvent(hs[s]->stream, halo[s + 1], 0);  // left-going halo of t-1
            rc = mrlbm_step_faces(hs[s]);
            if (rc != MRLBM_OK) break;
            cudaEventRecord(face[s], hs[s]->stream);
            rc = mrlbm_step(hs[s], 1, 0);
            cudaEventRecord(done[s], hs[s]->stream);
        }
        for (int s = 0; s < n && rc == MRLBM_OK; ++s) {
            cudaSetDevice(hs[s]->device);
            cudaStreamWaitEvent(side[s], face[s], 0);
            // after mrlbm_step the handles' current level is the one step t writes
            if (s > 0) rc = halo_copy(hs[s], 0, nullptr, true, hs[s - 1]->buf[hs[s - 1]->cur], hs[s - 1], false, side[s]);
            if (rc == MRLBM_OK && s + 1 < n)
                rc = halo_copy(hs[s], 1, nullptr, true, hs[s + 1]->buf[hs[s + 1]->cur], hs[s + 1], false, side[s]);
            cudaEventRecord(halo[s], side[s]);
        }
    }
    for (int s = 0; s < n; ++s) {
        if (!side[s]) continue;
        cudaSetDevice(hs[s]->device);
        cudaStreamWaitEvent(hs[s]->stream, halo[s], 0);
        if (s > 0) cudaStreamWaitEvent(hs[s]->stream, halo[s - 1], 0);
        if (s + 1 < n) cudaStreamWaitEvent(hs[s]->stream, halo[s + 1], 0);
    }
    for (int s = 0; s < n; ++s) {
        if (!side[s]) continue;
        cudaSetDevice(hs[s]->device);
        cudaStreamSynchronize(hs[s]->stream);
        cudaStreamSynchronize(side[s]);
        cudaStreamDestroy(side[s]);
        cudaEventDestroy(face[s]);
        cudaEventDestroy(done[s]);
        cudaEventDestroy(halo[s]);
    }
    return rc;
}

int mrlbm_destroy(mrlbm_handle* h) {
    if (!h) return MRLBM_OK;
    free_all(h);
    delete h;
    return MRLBM_OK;
}

int mrlbm_last_error(const mrlbm_handle* h, char* buf, size_t len) {
    if (!buf || len == 0) return MRLBM_EINVAL;
    const std::string& s = h ? h->err : g_create_error;
    std::snprintf(buf, len, "%s", s.c_str());
    return MRLBM_OK;
}

int mrlbm_status(mrlbm_handle* h) {
    if (!h) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    CK(cudaSetDevice(h->device));
    int e = 0;
    CK(cudaMemcpyAsync(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (e & 4) return fail(h, MRLBM_EDEVICE_TIMEOUT, "device flag: tensor-copy wait timed out");
    if (e) return fail(h, MRLBM_EDEVICE_NAN, "device flag: NaN or non-positive density");
    return MRLBM_OK;
}

int mrlbm_set_stream(mrlbm_handle* h, void* s) {
    if (!h) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    h->stream = (cudaStream_t)s;
    return MRLBM_OK;
}

int mrlbm_get_geometry_info(const mrlbm_handle* h, mrlbm_geometry_info* info) {
    if (!h || !info) return MRLBM_EINVAL;
    info->nx = h->L.nx; info->ny = h->L.ny; info->nbct = h->geo.nb; info->n_label15 = h->geo.n_label15;
    info->x_c = h->geo.x_c; info->y_c = h->geo.y_c; info->r_c = h->geo.r_c; info->r_cyl = h->geo.r_cyl;
    info->nu = h->nu; info->omega = h->omega;
    info->pitch = h->L.pitch; info->off = h->L.off; info->plane = h->L.plane;
    info->state_bytes = 2 * h->L.total() * (int64_t)h->elem;
    return MRLBM_OK;
}

int mrlbm_get_boundary_nodes(const mrlbm_handle* h, int32_t* bou_i, int32_t* bou_j, int32_t* label_bc,
                             double* delta_uk, double* ref_xy, int32_t* stencil) {
    if (!h) return MRLBM_EINVAL;
    const Geometry& g = h->geo;
    for (int l = 0; l < g.nb; ++l) {
        if (bou_i) bou_i[l] = g.bi[l];
        if (bou_j) bou_j[l] = g.bj[l];
        if (label_bc) label_bc[l] = g.label[l];
        if (delta_uk) delta_uk[l] = g.delta[l];
    }
    if (ref_xy) std::copy(g.ref.begin(), g.ref.end(), ref_xy);
    if (stencil) std::copy(g.sten.begin(), g.sten.end(), stencil);
    return MRLBM_OK;
}

int mrlbm_get_node_classes(const mrlbm_handle* h, int32_t* isfluid, int32_t* issolid, int32_t* isbound) {
    if (!h) return MRLBM_EINVAL;
    const size_t N = h->geo.cls.size();
    for (size_t n = 0; n < N; ++n) {
        const int c = h->geo.cls[n];
        if (isfluid) isfluid[n] = c == 0;
        if (issolid) issolid[n] = c == 1;
        if (isbound) isbound[n] = c == 2;
    }
    return MRLBM_OK;
}

int mrlbm_load_state(mrlbm_handle* h, const double* f, int32_t iter) {
    if (!h || !f) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    CK(cudaSetDevice(h->device));
    int rc = upload_state(h, f);
    if (rc != MRLBM_OK) return rc;
    h->iter = iter;
    return MRLBM_OK;
}

int mrlbm_get_state(mrlbm_handle* h, double* f) {
    if (!h || !f) return MRLBM_EINVAL;
    if (h->host_only) {                 // the configured initial populations
        std::vector<double> f0;
        initial_state(h->cfg, h->lat, h->L.nx, h->L.ny, f0);
        std::copy(f0.begin(), f0.end(), f);
        return MRLBM_OK;
    }
    CK(cudaSetDevice(h->device));
    const int nx = h->L.nx, ny = h->L.ny;
    const size_t N = (size_t)nx * ny;
    if (!h->d_fstage) CK(cudaMalloc((void**)&h->d_fstage, N * Q * sizeof(double)));
    const mrlbm_config& c = h->cfg;
    CK(launch_gather_state(h->precision, h->buf[h->cur], h->d_fstage, h->L, c.x_periodic != 0, c.y_periodic != 0,
                           c.wall_mode == MRLBM_WALL_FREESLIP && !c.y_periodic, h->lat.w, h->stream, h->halo_l, h->halo_r));
    ++h->launches;
    CK(cudaMemcpyAsync(f, h->d_fstage, N * Q * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (h->ovr_live)
        for (const OvrEntry& e : h->ovr)
            f[(size_t)(e.i - 1) + (size_t)nx * (e.j - 1) + N * e.k] =
                h->precision == MRLBM_FP64 ? e.v : h->lat.w[e.k] + e.v;
    return MRLBM_OK;
}

int mrlbm_set_inlet_profile(mrlbm_handle* h, const double* u_in) {
    if (!h) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    CK(cudaSetDevice(h->device));
    if (!u_in) { h->has_uin = false; return MRLBM_OK; }
    const int ny = h->L.ny;
    if (!h->d_uin) CK(cudaMalloc((void**)&h->d_uin, (size_t)ny * sizeof(double)));
    if (h->precision == MRLBM_FP64) {
        CK(cudaMemcpyAsync(h->d_uin, u_in, (size_t)ny * 8, cudaMemcpyHostToDevice, h->stream));
    } else {
        std::vector<float> t(u_in, u_in + ny);
        CK(cudaMemcpyAsync(h->d_uin, t.data(), (size_t)ny * 4, cudaMemcpyHostToDevice, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    h->has_uin = true;
    return MRLBM_OK;
}

int mrlbm_surface_enable(mrlbm_handle* h, int32_t enable) {
    if (!h) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    if (!enable) { h->surf_on = false; return MRLBM_OK; }
    const Geometry& g = h->geo;
    const int nb = g.nb;
    if (nb == 0) return fail(h, MRLBM_EUNSUPPORTED, "no cylinder: no surface to sample");
    if ((size_t)nb * sizeof(double) > 48 * 1024) return fail(h, MRLBM_EUNSUPPORTED, "more than 6144 wall nodes");
    const mrlbm_config& c = h->cfg;
    // probes (2d_mrlbm.f90:102-109): 1, 1.5, 2 and 2.5 diameters behind the centre, one row above it
    int pi[4], pj[4];
    if (c.geometry_mode == MRLBM_GEOM_REFERENCE) {
        const int nfront = c.L_front * c.ncy, nbot = c.L_bot * c.ncy, ncy = c.ncy;
        const int base = nfront + ncy + 1;
        pi[0] = base + ncy / 2; pi[1] = base + ncy; pi[2] = base + 3 * ncy / 2; pi[3] = base + 2 * ncy;
        for (int k = 0; k < 4; ++k) pj[k] = nbot + ncy / 2 + 1;
    } else {
        for (int k = 0; k < 4; ++k) {
            pi[k] = (int)std::floor(g.x_c + (1.0 + 0.5 * k) * 2.0 * g.r_c + 0.5);
            pj[k] = (int)std::floor(g.y_c) + 1;
        }
    }
    for (int k = 0; k < 4; ++k) {
        if (pi[k] < 1 || pi[k] > h->L.nx || pj[k] < 1 || pj[k] > h->L.ny)
            return fail(h, MRLBM_EUNSUPPORTED, "a probe falls outside the domain");
        if (g.cls[(size_t)(pi[k] - 1) + (size_t)h->L.nx * (pj[k] - 1)] != 0)
            return fail(h, MRLBM_EUNSUPPORTED, "a probe falls on a solid or wall node");
    }
    CK(cudaSetDevice(h->device));
    if (!h->d_quad) {
        // radii for quadratic_interpolation (2d_mrlbm.f90:742-765), points 2, 3, 4 and the wall point
        std::vector<double> quad(5 * (size_t)nb);
        auto rad = [](double x, double y) { return std::sqrt((x * x) + (y * y)); };
        for (int l = 0; l < nb; ++l) {
            const double* r = &g.ref[8 * (size_t)l];
            const double r1 = rad(r[1] - g.x_c, r[5] - g.y_c), r2 = rad(r[2] - g.x_c, r[6] - g.y_c);
            const double r3 = rad(r[3] - g.x_c, r[7] - g.y_c), rs = rad(r[0] - g.x_c, r[4] - g.y_c);
            double* q = &quad[5 * (size_t)l];
            q[0] = r1; q[1] = r2; q[2] = r3; q[3] = rs;
            q[4] = (r1 - r2) * (r1 - r3) * (r2 - r3);
        }
        // theta order by the reference's selection swap (2d_mrlbm.f90:1138-1156)
        std::vector<int> idx(nb);
        for (int i = 0; i < nb; ++i) idx[i] = i;
        for (int i = 0; i < nb - 1; ++i)
            for (int j = i + 1; j < nb; ++j)
                if (g.theta[idx[i]] > g.theta[idx[j]]) std::swap(idx[i], idx[j]);
        // Gaussian weights over the sorted angles (gaussian_smoothing, 2d_mrlbm.f90:718-740)
        std::vector<double> W((size_t)nb * nb), sumw(nb);
        const double sigma = 0.1;
        for (int i = 0; i < nb; ++i) {
            double sw = 0.0;
            for (int j = 0; j < nb; ++j) {
                const double d = g.theta[idx[i]] - g.theta[idx[j]];
                const double w = std::exp(-(d * d) / (2.0 * (sigma * sigma)));
                W[(size_t)j * nb + i] = w;
                sw = sw + w;
            }
            sumw[i] = sw;
        }
        h->surf_cap = (int)std::max<size_t>(1, std::min<size_t>(RING_CAP, ((size_t)64 << 20) / ((size_t)2 * nb * sizeof(double))));
        CK(cudaMalloc((void**)&h->d_quad, quad.size() * sizeof(double)));
        CK(cudaMalloc((void**)&h->d_sidx, nb * sizeof(int)));
        CK(cudaMalloc((void**)&h->d_W, W.size() * sizeof(double)));
        CK(cudaMalloc((void**)&h->d_sumw, nb * sizeof(double)));
        CK(cudaMalloc((void**)&h->d_sring, (size_t)h->surf_cap * 2 * nb * sizeof(double)));
        CK(cudaMalloc((void**)&h->d_pring, (size_t)h->surf_cap * 12 * sizeof(double)));
        CK(cudaMemcpyAsync(h->d_quad, quad.data(), quad.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->d_sidx, idx.data(), nb * sizeof(int), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->d_W, W.data(), W.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->d_sumw, sumw.data(), nb * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    h->surf.quad = h->d_quad;
    h->surf.idx = h->d_sidx;
    h->surf.W = h->d_W;
    h->surf.sumw = h->d_sumw;
    h->surf.nb = nb;
    for (int k = 0; k < 4; ++k) { h->surf.probe_i[k] = pi[k]; h->surf.probe_j[k] = pj[k]; }
    h->surf_on = true;
    return MRLBM_OK;
}

int mrlbm_get_probe_nodes(const mrlbm_handle* h, int32_t* pi, int32_t* pj) {
    if (!h || !pi || !pj || !h->surf_on) return MRLBM_EINVAL;
    for (int k = 0; k < 4; ++k) { pi[k] = h->surf.probe_i[k]; pj[k] = h->surf.probe_j[k]; }
    return MRLBM_OK;
}

int mrlbm_get_surface(mrlbm_handle* h, int32_t* iter, double* p_surface, double* p_smooth, double* probes,
                      int32_t cap, int32_t* n) {
    if (!h || !n || cap < 0) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    CK(cudaSetDevice(h->device));
    int rc = drain_surface(h);
    if (rc != MRLBM_OK) return rc;
    const int nb = h->geo.nb;
    const int m = std::min<int>(cap, (int)h->surf_iter.size());
    for (int r = 0; r < m; ++r) {
        if (iter) iter[r] = h->surf_iter[r];
        const double* src = h->surf_hist.data() + (size_t)r * 2 * nb;
        if (p_surface) std::memcpy(p_surface + (size_t)r * nb, src, nb * sizeof(double));
        if (p_smooth) std::memcpy(p_smooth + (size_t)r * nb, src + nb, nb * sizeof(double));
        if (probes) std::memcpy(probes + (size_t)r * 12, h->probe_hist.data() + (size_t)r * 12, 12 * sizeof(double));
    }
    h->surf_iter.erase(h->surf_iter.begin(), h->surf_iter.begin() + m);
    h->surf_hist.erase(h->surf_hist.begin(), h->surf_hist.begin() + (size_t)m * 2 * nb);
    h->probe_hist.erase(h->probe_hist.begin(), h->probe_hist.begin() + (size_t)m * 12);
    *n = m;
    return MRLBM_OK;
}

int mrlbm_set_body_force(mrlbm_handle* h, const double* g) {
    if (!h) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    CK(cudaSetDevice(h->device));
    if (!g) { h->has_body = false; return MRLBM_OK; }
    const size_t n2 = (size_t)2 * h->L.nx * h->L.ny;
    if (!h->d_body) CK(cudaMalloc(&h->d_body, n2 * h->elem));
    if (h->precision == MRLBM_FP64) {
        CK(cudaMemcpyAsync(h->d_body, g, n2 * 8, cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    } else {
        std::vector<float> t(g, g + n2);
        CK(cudaMemcpyAsync(h->d_body, t.data(), n2 * 4, cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    h->has_body = true;
    return MRLBM_OK;
}

int mrlbm_step(mrlbm_handle* h, int32_t nsteps, int32_t flags) {
    if (!h || nsteps < 0) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    CK(cudaSetDevice(h->device));
    const mrlbm_config& c = h->cfg;
    if ((flags & MRLBM_STEP_MACRO) && !h->d_macro)
        CK(cudaMalloc((void**)&h->d_macro, (size_t)6 * h->L.nx * h->L.ny * sizeof(double)));
    for (int s = 0; s < nsteps; ++s) {
        h->iter += 1;
        const bool stats = c.post_process && h->iter >= c.statsbegin && h->iter <= c.statsend;
        const bool plot = c.post_process && c.iplot > 0 && h->iter % c.iplot == 0 &&
                          (c.channel_with_cylinder || c.channel_with_square);
        const bool macro = (flags & MRLBM_STEP_MACRO) && s == nsteps - 1;
        int rc = launch_one(h, stats, plot, macro);
        if (rc != MRLBM_OK) {
            if (rc == MRLBM_EUNSUPPORTED) h->iter -= 1;      // nothing was launched
            return rc;
        }
        if (h->ring_n == RING_CAP) {
            rc = drain_ring(h);
            if (rc != MRLBM_OK) return rc;
        }
    }
    return MRLBM_OK;
}

int mrlbm_get_iter(const mrlbm_handle* h, int32_t* iter) {
    if (!h || !iter) return MRLBM_EINVAL;
    *iter = h->iter;
    return MRLBM_OK;
}

int mrlbm_field_stats_window(mrlbm_handle* h, int32_t begin_iter, int32_t end_iter) {
    if (!h || begin_iter > end_iter) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    CK(cudaSetDevice(h->device));
    const size_t bytes = (size_t)6 * h->L.nx * h->L.ny * sizeof(double);
    if (!h->d_fstat) {
        CK(cudaMalloc((void**)&h->d_fstat, bytes));
        CK(cudaMalloc((void**)&h->d_fstat_out, bytes));
    }
    CK(cudaMemsetAsync(h->d_fstat, 0, bytes, h->stream));
    h->fstat_begin = begin_iter;
    h->fstat_end = end_iter;
    h->fstat_n = 0;
    return MRLBM_OK;
}

int mrlbm_field_stats_get(mrlbm_handle* h, double* mean_u, double* mean_v, double* mean_p, double* rms_u,
                          double* rms_v, double* rms_p, int64_t* n_samples) {
    if (!h) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    if (!h->d_fstat) return fail(h, MRLBM_ESTATE, "no field-statistics window (mrlbm_field_stats_window)");
    if (n_samples) *n_samples = h->fstat_n;
    if (h->fstat_n == 0) return fail(h, MRLBM_ESTATE, "no step inside the field-statistics window yet");
    CK(cudaSetDevice(h->device));
    const int64_t N = (int64_t)h->L.nx * h->L.ny;
    CK(launch_field_stats_finalize(h->d_fstat, h->d_fstat_out, N, h->fstat_n, h->stream));
    ++h->launches;
    double* outs[6] = {mean_u, mean_v, mean_p, rms_u, rms_v, rms_p};
    for (int q = 0; q < 6; ++q)
        if (outs[q])
            CK(cudaMemcpyAsync(outs[q], h->d_fstat_out + q * N, N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MRLBM_OK;
}

int mrlbm_get_macro(mrlbm_handle* h, double* rho, double* ux, double* uy, double* mxx, double* myy, double* mxy) {
    if (!h) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    if (!h->d_macro) return fail(h, MRLBM_ESTATE, "no step has stored macroscopic fields (use MRLBM_STEP_MACRO)");
    CK(cudaSetDevice(h->device));
    const size_t N = (size_t)h->L.nx * h->L.ny;
    double* outs[6] = {rho, ux, uy, mxx, myy, mxy};
    for (int q = 0; q < 6; ++q)
        if (outs[q]) CK(cudaMemcpyAsync(outs[q], h->d_macro + q * N, N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MRLBM_OK;
}

int mrlbm_get_forces(mrlbm_handle* h, int32_t* iter, double* fd, double* fl, double* rin, int32_t cap, int32_t* n) {
    if (!h || !n) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    CK(cudaSetDevice(h->device));
    int rc = drain_ring(h);
    if (rc != MRLBM_OK) return rc;
    const int avail = (int)(h->hist.size() / REC_WORDS);
    const int m = std::min(avail, std::max(cap, 0));
    for (int t = 0; t < m; ++t) {
        const double* r = &h->hist[(size_t)t * REC_WORDS];
        if (iter) iter[t] = (int32_t)r[0];
        if (fd) fd[t] = r[1];
        if (fl) fl[t] = r[2];
        if (rin) rin[t] = r[3];
    }
    h->hist.erase(h->hist.begin(), h->hist.begin() + (size_t)m * REC_WORDS);
    *n = m;
    return MRLBM_OK;
}

int mrlbm_step_noalloc(mrlbm_handle* h, void* d_state, const double* d_f0, int32_t nsteps, double* records,
                       int32_t* n_records, void* stream) {
    if (!h || nsteps < 0) return MRLBM_EINVAL;
    if (!h->host_only) return fail(h, MRLBM_EINVAL, "mrlbm_step_noalloc takes a host-only handle (device -1)");
    const mrlbm_config& c = h->cfg;
    NaCase nc;
    nc.geo = &h->geo;
    nc.geo32 = &h->geo32;
    nc.precision = h->precision;
    nc.L = h->L;
    for (int k = 0; k < Q; ++k) nc.w[k] = h->lat.w[k];
    nc.xper = c.x_periodic != 0;
    nc.yper = c.y_periodic != 0;
    nc.freeslip = c.wall_mode == MRLBM_WALL_FREESLIP && !c.y_periodic;
    nc.post_process = c.post_process;
    nc.statsbegin = c.statsbegin;
    nc.statsend = c.statsend;
    nc.iplot = c.iplot;
    nc.plot_enabled = c.post_process && (c.channel_with_cylinder || c.channel_with_square);
    StepParams<double> p64{};
    StepParams<float> p32{};
    if (h->precision == MRLBM_FP64) { fill_common(h, p64); nc.p64 = &p64; }
    else { fill_common(h, p32); nc.p32 = &p32; }
    if (d_f0) nc.conflicts = slot_conflicts(h);
    nc.tile_cfg = is_tma_cfg(h->tile_cfg) ? 1 : h->tile_cfg;   // TMA shapes need handle-owned counters
    nc.iter = h->iter;
    nc.cur = h->cur;
    nc.launches = h->launches;
    std::string err;
    const int rc = noalloc_step(nc, d_state, d_f0, nsteps, records, n_records, stream, err);
    h->iter = nc.iter;
    h->cur = nc.cur;
    h->launches = nc.launches;
    if (rc != MRLBM_OK) h->err = err;
    return rc;
}

int mrlbm_set_tile_config(mrlbm_handle* h, int32_t cfg) {
    if (!h || cfg < 0 || cfg >= N_ALL_CFGS) return MRLBM_EINVAL;
    h->tile_cfg = cfg;
    return MRLBM_OK;
}

int mrlbm_get_tile_config(const mrlbm_handle* h, int32_t* cfg) {
    if (!h || !cfg) return MRLBM_EINVAL;
    *cfg = h->tile_cfg;
    return MRLBM_OK;
}

int mrlbm_autotune(mrlbm_handle* h, int32_t trial_steps, int32_t* best_cfg, double* best_ms) {
    if (!h || trial_steps < 1) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    CK(cudaSetDevice(h->device));
    int drc = drain_ring(h);                            // pending records go to the history first
    if (drc != MRLBM_OK) return drc;
    // everything a trial changes is saved and put back: both time levels, iteration, ring
    const size_t bytes = (size_t)h->L.total() * h->elem;
    void* save[2] = {nullptr, nullptr};
    CK(cudaMalloc(&save[0], bytes));
    if (cudaMalloc(&save[1], bytes) != cudaSuccess) {
        cudaFree(save[0]);
        return fail(h, MRLBM_ECUDA, "cudaMalloc autotune save");
    }
    auto cleanup = [&]() { cudaFree(save[0]); cudaFree(save[1]); };
    const int iter0 = h->iter, cur0 = h->cur, ring0 = h->ring_n;
    const bool ovr0 = h->ovr_live;
    const size_t hist0 = h->hist.size();
    // trials record no surface pressure; with a field-statistics window the trials accumulate
    // too (the choice fits that workload) into sums saved here and put back afterwards
    const bool surf0 = h->surf_on;
    const int32_t fsb0 = h->fstat_begin, fse0 = h->fstat_end;
    const int64_t fsn0 = h->fstat_n;
    const size_t fbytes = (size_t)6 * h->L.nx * h->L.ny * sizeof(double);
    double* fsave = nullptr;
    h->surf_on = false;
    if (h->d_fstat) {
        if (cudaMalloc((void**)&fsave, fbytes) != cudaSuccess ||
            cudaMemcpyAsync(fsave, h->d_fstat, fbytes, cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess) {
            if (fsave) cudaFree(fsave);
            fsave = nullptr;
            h->fstat_begin = 1;                        // no room to save the sums: trials without them
            h->fstat_end = 0;
        } else {
            h->fstat_begin = std::numeric_limits<int32_t>::min();
            h->fstat_end = std::numeric_limits<int32_t>::max();
        }
    }
    for (int b = 0; b < 2; ++b)
        if (cudaMemcpyAsync(save[b], h->buf[b], bytes, cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess) {
            h->surf_on = surf0;
            h->fstat_begin = fsb0;
            h->fstat_end = fse0;
            if (fsave) cudaFree(fsave);
            cleanup();
            return fail(h, MRLBM_ECUDA, "autotune save copy");
        }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int cfg0 = h->tile_cfg;
    int best = cfg0;
    float best_t = 1e30f;
    int rc = MRLBM_OK;
    for (int c = 0; c < N_ALL_CFGS && rc == MRLBM_OK; ++c) {
        h->tile_cfg = c;
        rc = mrlbm_step(h, 1, 0);                       // warm-up (and instruction cache)
        if (rc == MRLBM_EUNSUPPORTED) {                 // shape does not fit: nothing ran
            rc = MRLBM_OK;
            h->iter = iter0;
            continue;
        }
        if (rc != MRLBM_OK) break;
        cudaEventRecord(e0, h->stream);
        rc = mrlbm_step(h, trial_steps, 0);
        cudaEventRecord(e1, h->stream);
        if (rc != MRLBM_OK || cudaEventSynchronize(e1) != cudaSuccess) { rc = rc ? rc : MRLBM_ECUDA; break; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_t) { best_t = ms; best = c; }
        // restore before the next trial so every shape starts from the same state
        for (int b = 0; b < 2; ++b)
            if (cudaMemcpyAsync(h->buf[b], save[b], bytes, cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess)
                rc = MRLBM_ECUDA;
        h->iter = iter0;
        h->cur = cur0;
        h->ring_n = ring0;
        h->ovr_live = ovr0;
        h->hist.resize(hist0);
        h->pend.on = false;                             // the trials' last record is discarded
    }
    h->surf_on = surf0;
    h->fstat_begin = fsb0;
    h->fstat_end = fse0;
    h->fstat_n = fsn0;
    if (fsave) {
        cudaMemcpyAsync(h->d_fstat, fsave, fbytes, cudaMemcpyDeviceToDevice, h->stream);
        cudaStreamSynchronize(h->stream);
        cudaFree(fsave);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamSynchronize(h->stream);
    cleanup();
    if (rc != MRLBM_OK) {
        h->tile_cfg = cfg0;
        return rc;
    }
    h->tile_cfg = best;
    if (best_cfg) *best_cfg = best;
    if (best_ms) *best_ms = best_t / trial_steps;
    return MRLBM_OK;
}

int mrlbm_get_launch_count(const mrlbm_handle* h, int64_t* n) {
    if (!h || !n) return MRLBM_EINVAL;
    *n = h->launches;
    return MRLBM_OK;
}

}  // extern "C"


// ---- adjoint of the mean drag -------------------------------------------------------------

namespace {

// One forward step from src into dst at iteration `iter` (drag record into rec if given).
template <class T>
int adj_forward(mrlbm_handle* h, const void* src, void* dst, int iter, double* rec, bool ovr, int tile, cudaStream_t st) {
    StepParams<T> p{};
    fill_common(h, p);
    const mrlbm_config& c = h->cfg;
    p.src = (const T*)src;
    p.dst = (T*)dst;
    p.u_in = h->has_uin ? (const T*)h->d_uin : nullptr;
    p.body = h->has_body ? (const T*)h->d_body : nullptr;
    p.ovr = ovr ? h->d_ovr : nullptr;
    p.n_ovr = ovr ? (int)h->ovr.size() : 0;
    p.zero_solid_u = c.post_process && c.iplot > 0 && iter % c.iplot == 0 && (c.channel_with_cylinder || c.channel_with_square);
    p.do_stats = rec != nullptr;
    p.rec = rec;
    p.iter = iter;
    h->launches += step_launches(sizeof(T) == 4, tile);
    if (sizeof(T) == 8) return launch_step_f64(reinterpret_cast<const StepParams<double>&>(p), tile, st, 0);
    return launch_step_f32(reinterpret_cast<const StepParams<float>&>(p), tile, st, 0);
}

template <class T>
int adj_backward(mrlbm_handle* h, const void* src, int iter, bool ovr, const adj::AdjArgs& a) {
    StepParams<T> p{};
    fill_common(h, p);
    const mrlbm_config& c = h->cfg;
    p.src = (const T*)src;
    p.u_in = h->has_uin ? (const T*)h->d_uin : nullptr;
    p.body = h->has_body ? (const T*)h->d_body : nullptr;
    p.ovr = ovr ? h->d_ovr : nullptr;
    p.n_ovr = ovr ? (int)h->ovr.size() : 0;
    p.zero_solid_u = c.post_process && c.iplot > 0 && iter % c.iplot == 0 && (c.channel_with_cylinder || c.channel_with_square);
    p.iter = iter;
    h->launches += 2;
    return launch_adjoint_step(p, a, h->stream);
}

}  // namespace

extern "C" int mrlbm_adjoint_drag(mrlbm_handle* h, int32_t nsteps, int32_t window, int32_t checkpoint_every,
                                  double* J, double* grad_body, double* grad_uin) {
    if (!h || nsteps < 1 || window < 1 || window > nsteps || checkpoint_every < 1 || !J) return MRLBM_EINVAL;
    if (h->host_only) return fail(h, MRLBM_ENODEVICE, "host-only handle (created with device -1)");
    const mrlbm_config& c = h->cfg;
    if (c.x_periodic || h->halo_l || h->halo_r)
        return fail(h, MRLBM_EUNSUPPORTED, "adjoint: needs inlet/outlet columns and a whole (not x-slab) lattice");
    const bool walls_ref = c.wall_mode == MRLBM_WALL_REFERENCE && !c.y_periodic;
    CK(cudaSetDevice(h->device));
    int rc = drain_ring(h);
    if (rc != MRLBM_OK) return rc;
    const int N = nsteps, K = std::min(checkpoint_every, nsteps), T = window;
    const int ncp = (N + K - 1) / K;
    const size_t LB = (size_t)h->L.total() * h->elem;            // a population level
    const size_t LAM = (size_t)h->L.total() * sizeof(double);     // an adjoint level (FP64)
    const bool fp64 = h->precision == MRLBM_FP64;
    const int64_t nodes = (int64_t)h->L.nx * h->L.ny;
    const int tile = is_tma_cfg(h->tile_cfg) ? 1 : h->tile_cfg;
    const bool grads = grad_body || grad_uin;
    std::vector<void*> cp(ncp, nullptr), seg(grads ? K : 0, nullptr), seg2(grads ? K : 0, nullptr);
    void* work[2] = {nullptr, nullptr};
    double *lam[2] = {nullptr, nullptr}, *d_rec = nullptr, *gb = nullptr, *gu = nullptr;
    // One workspace for the checkpoints, two sets of segment levels (one replayed, one being
    // recomputed), two working levels, the drag records and the adjoint fields, kept with the
    // handle so repeated calls (a gradient loop) allocate nothing; it grows when a call needs more.
    const auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t n_levels = (size_t)ncp + (seg.empty() ? 0 : 2 * (seg.size() - 1)) + 2;
    const size_t ws = n_levels * al(LB) + al((size_t)N * REC_WORDS * sizeof(double)) + al(sizeof(unsigned)) +
                      (grads ? 2 * al(LAM) + al((size_t)2 * nodes * sizeof(double)) + al((size_t)h->L.ny * sizeof(double)) : 0);
    if (h->adj_ws_bytes < ws) {
        if (h->adj_ws) cudaFree(h->adj_ws);
        h->adj_ws = nullptr;
        h->adj_ws_bytes = 0;
        if (cudaMalloc(&h->adj_ws, ws) != cudaSuccess) {
            cudaGetLastError();
            return fail(h, MRLBM_ECUDA, "adjoint: device memory for checkpoints and adjoint fields");
        }
        h->adj_ws_bytes = ws;
    }
    char* wp = (char*)h->adj_ws;
    auto carve = [&](size_t b) { void* q = wp; wp += al(b); return q; };
    bool ok = true;
    auto level = [&](void** q) {
        *q = carve(LB);
        // every level carries the never-written ghost values of the current state
        return cudaMemcpyAsync(*q, h->buf[h->cur], LB, cudaMemcpyDeviceToDevice, h->stream) == cudaSuccess;
    };
    for (int q = 0; q < ncp && ok; ++q) ok = level(&cp[q]);
    for (int q = 1; q < (int)seg.size() && ok; ++q) ok = level(&seg[q]) && level(&seg2[q]);   // [0] borrows a checkpoint
    ok = ok && level(&work[0]) && level(&work[1]);
    d_rec = (double*)carve((size_t)N * REC_WORDS * sizeof(double));
    unsigned* d_done = (unsigned*)carve(sizeof(unsigned));      // the adjoint bulk launches' counter
    ok = ok && cudaMemsetAsync(d_done, 0, sizeof(unsigned), h->stream) == cudaSuccess;
    if (ok && grads) {
        lam[0] = (double*)carve(LAM);
        lam[1] = (double*)carve(LAM);
        gb = (double*)carve((size_t)2 * nodes * sizeof(double));
        gu = (double*)carve((size_t)h->L.ny * sizeof(double));
        ok = cudaMemsetAsync(lam[0], 0, LAM, h->stream) == cudaSuccess &&
             cudaMemsetAsync(lam[1], 0, LAM, h->stream) == cudaSuccess &&
             cudaMemsetAsync(gb, 0, (size_t)2 * nodes * sizeof(double), h->stream) == cudaSuccess &&
             cudaMemsetAsync(gu, 0, (size_t)h->L.ny * sizeof(double), h->stream) == cudaSuccess;
    }
    auto release = [&]() {};                                       // the workspace stays with the handle
    if (!ok) {
        cudaGetLastError();
        return fail(h, MRLBM_ECUDA, "adjoint: initialising checkpoints and adjoint fields");
    }
    const int it0 = h->iter;
    // forward pass: F^0 .. F^N, checkpoint F^{cK}, drag records of the window
    auto fwd = [&](const void* a, void* b, int it, double* rec, bool ovr, cudaStream_t st) {
        return fp64 ? adj_forward<double>(h, a, b, it, rec, ovr, tile, st) : adj_forward<float>(h, a, b, it, rec, ovr, tile, st);
    };
    const void* prev = cp[0];
    for (int n = 1; n <= N && rc == MRLBM_OK; ++n) {
        void* dst = work[n & 1];
        double* rec = n > N - T ? d_rec + (size_t)(n - 1) * REC_WORDS : nullptr;
        if (fwd(prev, dst, it0 + n, rec, n == 1 && h->ovr_live, h->stream) != 0) rc = MRLBM_ECUDA;
        if (n % K == 0 && n / K < ncp && cudaMemcpyAsync(cp[n / K], dst, LB, cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess)
            rc = MRLBM_ECUDA;
        prev = dst;
    }
    std::vector<double> recs((size_t)N * REC_WORDS);
    if (rc == MRLBM_OK &&
        (cudaMemcpyAsync(recs.data(), d_rec, recs.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
         cudaStreamSynchronize(h->stream) != cudaSuccess))
        rc = MRLBM_ECUDA;
    if (rc == MRLBM_OK) {
        double acc = 0.0;
        for (int n = N - T + 1; n <= N; ++n) acc = acc + recs[(size_t)(n - 1) * REC_WORDS + 1];
        *J = acc / T;
    }
    // Backward pass, segment by segment from the last checkpoint.  Segment c is recomputed from
    // checkpoint c into one of two buffer sets on a second stream while the adjoint kernels
    // sweep segment c + 1 from the other set on the handle's stream: a recompute waits for the
    // sweep that last used its set, a sweep for the recompute of its segment.
    std::vector<void*>* sets[2] = {&seg, &seg2};
    int sx0 = h->L.nx + 1, sx1 = 0, sy0 = h->L.ny + 1, sy1 = 0;   // stencil-node bounding box
    for (int l = 0; l < h->geo.nb; ++l)
        for (int m = 0; m < 12; ++m) {
            const int si = h->geo.tint[(size_t)(I_SI + m) * h->geo.nb + l], sj = h->geo.tint[(size_t)(I_SJ + m) * h->geo.nb + l];
            sx0 = std::min(sx0, si); sx1 = std::max(sx1, si); sy0 = std::min(sy0, sj); sy1 = std::max(sy1, sj);
        }
    cudaStream_t rs = nullptr;
    cudaEvent_t rec_done[2] = {nullptr, nullptr}, adj_done[2] = {nullptr, nullptr};
    if (grads && rc == MRLBM_OK) {
        bool made = cudaStreamCreateWithFlags(&rs, cudaStreamNonBlocking) == cudaSuccess;
        for (int q = 0; q < 2 && made; ++q)
            made = cudaEventCreateWithFlags(&rec_done[q], cudaEventDisableTiming) == cudaSuccess &&
                   cudaEventCreateWithFlags(&adj_done[q], cudaEventDisableTiming) == cudaSuccess;
        if (!made) rc = MRLBM_ECUDA;
    }
    auto recompute = [&](int cs, cudaStream_t st) {
        std::vector<void*>& sg = *sets[cs & 1];
        const int n0 = cs * K, m = std::min(K, N - n0);
        sg[0] = cp[cs];
        for (int t = 1; t < m; ++t)
            if (fwd(sg[t - 1], sg[t], it0 + n0 + t, nullptr, n0 + t == 1 && h->ovr_live, st) != 0) return MRLBM_ECUDA;
        return (int)MRLBM_OK;
    };
    if (grads && rc == MRLBM_OK) rc = recompute(ncp - 1, h->stream);
    int li = 0;
    for (int cseg = ncp - 1; grads && cseg >= 0 && rc == MRLBM_OK; --cseg) {
        const int n0 = cseg * K, m = std::min(K, N - n0);
        std::vector<void*>& sg = *sets[cseg & 1];
        if (cseg >= 1) {                                   // the next segment, meanwhile
            if (cseg + 1 <= ncp - 1) cudaStreamWaitEvent(rs, adj_done[(cseg + 1) & 1], 0);
            rc = recompute(cseg - 1, rs);
            if (rc == MRLBM_OK && cudaEventRecord(rec_done[(cseg - 1) & 1], rs) != cudaSuccess) rc = MRLBM_ECUDA;
        }
        if (cseg < ncp - 1) cudaStreamWaitEvent(h->stream, rec_done[cseg & 1], 0);
        for (int n = n0 + m; n > n0 && rc == MRLBM_OK; --n) {
            const int t = n - n0 - 1;                  // sg[t] = F^{n-1}
            adj::AdjArgs a{};
            a.lam_in = lam[li];
            a.lam_out = lam[li ^ 1];
            a.grad_body = gb;
            a.grad_uin = gu;
            a.wJ = n > N - T ? 1.0 / T : 0.0;
            a.n_edge = 2 * h->L.ny + (walls_ref ? 2 * (h->L.nx - 2) : 0);
            a.done = d_done;
            a.sx0 = sx0; a.sx1 = sx1; a.sy0 = sy0; a.sy1 = sy1;
            const bool ovr = n == 1 && h->ovr_live;
            if ((fp64 ? adj_backward<double>(h, sg[t], it0 + n, ovr, a) : adj_backward<float>(h, sg[t], it0 + n, ovr, a)) != 0)
                rc = MRLBM_ECUDA;
            li ^= 1;
        }
        if (rc == MRLBM_OK && cudaEventRecord(adj_done[cseg & 1], h->stream) != cudaSuccess) rc = MRLBM_ECUDA;
    }
    if (rc == MRLBM_OK && grads) {
        if (grad_body && cudaMemcpyAsync(grad_body, gb, (size_t)2 * nodes * sizeof(double), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
            rc = MRLBM_ECUDA;
        if (grad_uin && cudaMemcpyAsync(grad_uin, gu, (size_t)h->L.ny * sizeof(double), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
            rc = MRLBM_ECUDA;
    }
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) rc = MRLBM_ECUDA;
    if (rs) {
        if (cudaStreamSynchronize(rs) != cudaSuccess) rc = MRLBM_ECUDA;
        cudaStreamDestroy(rs);
    }
    for (int q = 0; q < 2; ++q) {
        if (rec_done[q]) cudaEventDestroy(rec_done[q]);
        if (adj_done[q]) cudaEventDestroy(adj_done[q]);
    }
    release();
    if (rc != MRLBM_OK) return fail(h, rc, std::string("adjoint: ") + cudaGetErrorString(cudaGetLastError()));
    return MRLBM_OK;
}

// ---- batched cases ----------------------------------------------------------------------

struct mrlbm_batch {
    std::vector<mrlbm_handle*> h;
    int precision = MRLBM_FP64, device = 0;
    cudaStream_t stream = nullptr;
    int tile_cfg = VEC_CFG0 + 2;
    int schedule = MRLBM_BATCH_PERSISTENT;
    int steps_per_launch = 64;
    int num_sms = 0;
    int64_t launches = 0;
    std::string err;
    void* d_params = nullptr;          // ncases x StepParams<T>
    BatchCase* d_cases = nullptr;
    int* d_off = nullptr;              // aux_off[n + 1], tile_off[n + 1]
    int* d_item_case = nullptr;        // case of each work item, for tile shape item_case_cfg
    size_t item_case_cap = 0;
    int item_case_cfg = -1;
    BatchBarrier* d_bar = nullptr;
    unsigned char* h_stage[2] = {nullptr, nullptr};   // pinned upload staging, double-buffered
    cudaEvent_t staged[2] = {nullptr, nullptr};
    int stage_i = 0;
    size_t stage_bytes = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_cfg = -1, graph_steps = 0, graph_macro = -1, graph_full = -1;
    unsigned wait_limit = BAR_SPIN_LIMIT;   // grid-barrier polls before a block gives up
    // Per-case streams schedule: every case's own step launches (the single-case kernels, with
    // their parameters in the constant bank) on a stream of its own, steps_per_launch steps per
    // case captured once into one graph (forked from and joined back into the batch stream) and
    // replayed; the record fields of each replay come from the call state uploaded before it.
    std::vector<cudaStream_t> cstream;
    std::vector<cudaEvent_t> join_ev;
    cudaEvent_t fork_ev = nullptr, call_staged = nullptr;
    int* d_call = nullptr;             // [2 n] iter0, ring_n0 of each case for the current replay
    int* h_call = nullptr;             // pinned staging of d_call
    struct StreamsGraph {
        cudaGraphExec_t exec = nullptr;
        int cfg = -1, steps = 0;
        std::vector<uintptr_t> sig;    // per case: time level, inlet-profile and body-force buffers when captured
    } sg[2];
    int sg_next = 0;
};

namespace {

int bfail(mrlbm_batch* b, int code, const std::string& msg) {
    b->err = msg;
    return code;
}

#define BCK(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) return bfail(b, MRLBM_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int stats_in(const mrlbm_config& c, int a, int z) {
    if (!c.post_process) return 0;
    const int lo = std::max(a, c.statsbegin), hi = std::min(z, c.statsend);
    return hi >= lo ? hi - lo + 1 : 0;
}

// Work items of one step of case h for vector shape cfg.
// Work items of one step of case h: auxiliary blocks of aux_threads threads, and the bulk tiles
// of shape cfg (a vector shape, or for split steps also a one-tile-per-block shape).
void batch_items(const mrlbm_handle* h, int cfg, int aux_threads, int& aux, int& tiles, int& nbblk, int& neblk,
                 int& tiles_x) {
    const int bn = aux_threads / 8;
    nbblk = h->geo.nb > 0 ? (h->geo.nb + bn - 1) / bn : 1;
    neblk = (2 * h->L.nx + (h->halo_l ? 0 : h->L.ny - 2) + (h->halo_r ? 0 : h->L.ny - 2) + aux_threads - 1) / aux_threads;
    int tiles_y;
    if (is_vec_cfg(cfg)) {
        const VecCfg v = VEC_CFGS[cfg - VEC_CFG0];
        const int vw = 16 / h->elem;
        tiles_x = (h->L.nx + 32 * vw - 1) / (32 * vw);
        tiles_y = (h->L.ny + v.warps * v.nj - 1) / (v.warps * v.nj);
    } else {
        const TileCfg t = TILE_CFGS[cfg];
        tiles_x = (h->L.nx + t.bx - 1) / t.bx;
        tiles_y = (h->L.ny + t.by * t.nj - 1) / (t.by * t.nj);
    }
    aux = nbblk + neblk;
    tiles = tiles_x * tiles_y;
}

// Split steps (the graph schedule) run the auxiliary items in blocks of their own size.
bool batch_split(const mrlbm_batch* b) { return b->schedule == MRLBM_BATCH_GRAPH || b->schedule == MRLBM_BATCH_STREAMS; }
int batch_aux_threads(const mrlbm_batch* b) {
    return batch_split(b) ? BATCH_AUX_THREADS : VEC_CFGS[b->tile_cfg - VEC_CFG0].warps * 32;
}

template <class T>
void batch_fill(mrlbm_batch* b, unsigned char* stage, int want_macro) {
    const int n = (int)b->h.size();
    StepParams<T>* ps = reinterpret_cast<StepParams<T>*>(stage);
    BatchCase* cs = reinterpret_cast<BatchCase*>(stage + n * sizeof(StepParams<T>));
    int* off = reinterpret_cast<int*>(stage + n * (sizeof(StepParams<T>) + sizeof(BatchCase)));
    int aux_acc = 0, tile_acc = 0;
    for (int c = 0; c < n; ++c) {
        mrlbm_handle* h = b->h[c];
        StepParams<T> p{};
        fill_common(h, p);
        p.src = (const T*)h->buf[h->cur];
        p.dst = (T*)h->buf[1 - h->cur];
        p.u_in = h->has_uin ? (const T*)h->d_uin : nullptr;
        p.body = h->has_body ? (const T*)h->d_body : nullptr;
        p.ovr = h->ovr_live ? h->d_ovr : nullptr;
        p.n_ovr = h->ovr_live ? (int)h->ovr.size() : 0;
        int aux, tiles;
        batch_items(h, b->tile_cfg, batch_aux_threads(b), aux, tiles, p.nbblk, p.neblk, p.tiles_x);
        p.tx_magic = tile_div_magic(p.tiles_x, tiles);
        ps[c] = p;
        BatchCase bc{};
        const mrlbm_config& k = h->cfg;
        bc.iter0 = h->iter;
        bc.cur0 = h->cur;
        bc.ring_n0 = h->ring_n;
        bc.ovr_live = h->ovr_live ? 1 : 0;
        bc.post_process = k.post_process != 0;
        bc.statsbegin = k.statsbegin;
        bc.statsend = k.statsend;
        bc.iplot = k.iplot;
        bc.plot_cyl = (k.channel_with_cylinder || k.channel_with_square) ? 1 : 0;
        bc.fs_begin = h->d_fstat ? h->fstat_begin : 1;
        bc.fs_end = h->d_fstat ? h->fstat_end : 0;
        bc.aux_items = aux;
        bc.tiles = tiles;
        bc.ring = h->d_ring;
        bc.macro = want_macro ? h->d_macro : nullptr;
        bc.fstat = h->d_fstat;
        cs[c] = bc;
        off[c] = aux_acc;
        off[n + 1 + c] = tile_acc;
        aux_acc += aux;
        tile_acc += tiles;
    }
    off[n] = aux_acc;
    off[2 * n + 1] = tile_acc;
}

size_t batch_param_bytes(const mrlbm_batch* b) {
    const size_t n = b->h.size();
    const size_t pb = b->precision == MRLBM_FP64 ? sizeof(StepParams<double>) : sizeof(StepParams<float>);
    return n * (pb + sizeof(BatchCase)) + (2 * n + 2) * sizeof(int);
}

// Whether a call of `steps` steps can replay captured single-case launches: a tile shape, and no
// step of it whose launch would differ from its captured form in more than the record fields
// (macroscopic output, field statistics, loaded-state overrides).  Other calls take the split
// graph schedule.
bool streams_call_ok(const mrlbm_batch* b, int steps, int want_macro) {
    if (b->tile_cfg < 0 || b->tile_cfg >= N_TILE_CFGS || want_macro) return false;
    for (const mrlbm_handle* h : b->h) {
        const mrlbm_config& c = h->cfg;
        const int a0 = h->iter + 1, z = h->iter + steps;
        if (h->ovr_live) return false;
        if (h->d_fstat && std::max(a0, h->fstat_begin) <= std::min(z, h->fstat_end)) return false;
    }
    return true;
}

template <class T>
int streams_launch_case(mrlbm_batch* b, int c, int steps) {
    mrlbm_handle* h = b->h[c];
    const mrlbm_config& k = h->cfg;
    StepParams<T> p{};
    fill_common(h, p);
    p.u_in = h->has_uin ? (const T*)h->d_uin : nullptr;
    p.body = h->has_body ? (const T*)h->d_body : nullptr;
    p.call = b->d_call + 2 * c;
    p.stats_lo = k.post_process ? k.statsbegin : 1;
    p.stats_hi = k.post_process ? k.statsend : 0;
    p.ring = h->d_ring;
    p.plot_every = k.post_process && k.iplot > 0 && (k.channel_with_cylinder || k.channel_with_square) ? k.iplot : 0;
    int cur = h->cur;
    for (int s = 0; s < steps; ++s) {
        p.src = (const T*)h->buf[cur];
        p.dst = (T*)h->buf[1 - cur];
        p.bstep = s;
        const int rc = sizeof(T) == 8 ? launch_step_f64(reinterpret_cast<const StepParams<double>&>(p), b->tile_cfg, b->cstream[c], 0)
                                      : launch_step_f32(reinterpret_cast<const StepParams<float>&>(p), b->tile_cfg, b->cstream[c], 0);
        if (rc != 0) return rc;
        cur ^= 1;
    }
    return 0;
}

int batch_call_streams(mrlbm_batch* b, int steps) {
    const int n = (int)b->h.size();
    const bool fp64 = b->precision == MRLBM_FP64;
    if (b->cstream.empty()) {                          // the per-case streams, once
        b->cstream.assign(n, nullptr);
        b->join_ev.assign(n, nullptr);
        for (int c = 0; c < n; ++c) {
            BCK(cudaStreamCreateWithFlags(&b->cstream[c], cudaStreamNonBlocking));
            BCK(cudaEventCreateWithFlags(&b->join_ev[c], cudaEventDisableTiming));
        }
        BCK(cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming));
        BCK(cudaEventCreateWithFlags(&b->call_staged, cudaEventDisableTiming));
        BCK(cudaMalloc((void**)&b->d_call, sizeof(int) * 2 * n));
        BCK(cudaMallocHost((void**)&b->h_call, sizeof(int) * 2 * n));
        BCK(cudaEventRecord(b->call_staged, b->stream));
    }
    for (mrlbm_handle* h : b->h) {
        int rc = finish_pending(h);
        if (rc == MRLBM_OK && h->ring_n + stats_in(h->cfg, h->iter + 1, h->iter + steps) > RING_CAP) rc = drain_ring(h);
        if (rc != MRLBM_OK) return bfail(b, rc, h->err);
    }
    // the call state, uploaded ahead of the replay on the batch stream
    BCK(cudaEventSynchronize(b->call_staged));
    for (int c = 0; c < n; ++c) {
        b->h_call[2 * c] = b->h[c]->iter;
        b->h_call[2 * c + 1] = b->h[c]->ring_n;
    }
    BCK(cudaMemcpyAsync(b->d_call, b->h_call, sizeof(int) * 2 * n, cudaMemcpyHostToDevice, b->stream));
    BCK(cudaEventRecord(b->call_staged, b->stream));
    // the graph captured for these cases' time levels (two are kept: an odd call length
    // alternates them)
    std::vector<uintptr_t> sig(3 * (size_t)n);
    for (int c = 0; c < n; ++c) {
        const mrlbm_handle* h = b->h[c];
        sig[3 * c] = (uintptr_t)h->cur;
        sig[3 * c + 1] = h->has_uin ? (uintptr_t)h->d_uin : 0;
        sig[3 * c + 2] = h->has_body ? (uintptr_t)h->d_body : 0;
    }
    mrlbm_batch::StreamsGraph* g = nullptr;
    for (auto& q : b->sg)
        if (q.exec && q.cfg == b->tile_cfg && q.steps == steps && q.sig == sig) g = &q;
    if (!g) {
        g = &b->sg[b->sg_next];
        b->sg_next ^= 1;
        if (g->exec) cudaGraphExecDestroy(g->exec);
        g->exec = nullptr;
        BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int rc = cudaEventRecord(b->fork_ev, b->stream) == cudaSuccess ? 0 : -1;
        for (int c = 0; c < n && rc == 0; ++c) {
            if (cudaStreamWaitEvent(b->cstream[c], b->fork_ev, 0) != cudaSuccess) { rc = -1; break; }
            rc = fp64 ? streams_launch_case<double>(b, c, steps) : streams_launch_case<float>(b, c, steps);
            // every forked stream is joined back, also after a failed launch, so that ending the
            // capture leaves no stream in capture mode
            const bool joined = cudaEventRecord(b->join_ev[c], b->cstream[c]) == cudaSuccess &&
                                cudaStreamWaitEvent(b->stream, b->join_ev[c], 0) == cudaSuccess;
            if (rc == 0 && !joined) rc = -1;
        }
        cudaGraph_t gr = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->stream, &gr);
        if (rc != 0 || e != cudaSuccess) {
            if (gr) cudaGraphDestroy(gr);
            cudaGetLastError();
            return bfail(b, rc == -2 ? MRLBM_EUNSUPPORTED : MRLBM_ECUDA, "capturing the per-case streams graph failed");
        }
        e = cudaGraphInstantiate(&g->exec, gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) return bfail(b, MRLBM_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        g->cfg = b->tile_cfg;
        g->steps = steps;
        g->sig = sig;
    }
    BCK(cudaGraphLaunch(g->exec, b->stream));
    for (mrlbm_handle* h : b->h) {
        h->ring_n += stats_in(h->cfg, h->iter + 1, h->iter + steps);
        h->iter += steps;
        h->cur ^= steps & 1;
        b->launches += (int64_t)steps * step_launches(!fp64, b->tile_cfg);
    }
    return MRLBM_OK;
}

// One call of `steps` steps (at most RING_CAP stats records per case).
int batch_call(mrlbm_batch* b, int steps, int want_macro) {
    const int n = (int)b->h.size();
    for (int c = 0; c < n; ++c)
        if (b->h[c]->surf_on)
            return bfail(b, MRLBM_EUNSUPPORTED, "case " + std::to_string(c) +
                                                    ": surface-pressure records are taken by single-case steps only");
    if (b->schedule == MRLBM_BATCH_STREAMS && streams_call_ok(b, steps, want_macro)) return batch_call_streams(b, steps);
    for (mrlbm_handle* h : b->h) {
        if (h->ring_n + stats_in(h->cfg, h->iter + 1, h->iter + steps) > RING_CAP) {
            int rc = drain_ring(h);
            if (rc != MRLBM_OK) return bfail(b, rc, h->err);
        }
        if (want_macro && !h->d_macro)
            BCK(cudaMalloc((void**)&h->d_macro, (size_t)6 * h->L.nx * h->L.ny * sizeof(double)));
    }
    // stage the per-call parameters in pinned memory and upload them
    const int si = b->stage_i;
    BCK(cudaEventSynchronize(b->staged[si]));
    if (b->precision == MRLBM_FP64) batch_fill<double>(b, b->h_stage[si], want_macro);
    else batch_fill<float>(b, b->h_stage[si], want_macro);
    const size_t pb = (b->precision == MRLBM_FP64 ? sizeof(StepParams<double>) : sizeof(StepParams<float>)) * n;
    const size_t cb = sizeof(BatchCase) * n;
    BCK(cudaMemcpyAsync(b->d_params, b->h_stage[si], pb, cudaMemcpyHostToDevice, b->stream));
    BCK(cudaMemcpyAsync(b->d_cases, b->h_stage[si] + pb, cb, cudaMemcpyHostToDevice, b->stream));
    BCK(cudaMemcpyAsync(b->d_off, b->h_stage[si] + pb + cb, (2 * n + 2) * sizeof(int), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaEventRecord(b->staged[si], b->stream));
    b->stage_i ^= 1;
    const int* off = reinterpret_cast<const int*>(b->h_stage[si] + pb + cb);
    const int items = off[n] + off[2 * n + 1];
    const int table_key = 2 * b->tile_cfg + (batch_split(b) ? 1 : 0);
    if (b->item_case_cfg != table_key) {               // the item -> case table of this shape and schedule
        std::vector<int> tab((size_t)items);
        for (int c = 0; c < n; ++c) {
            for (int k = off[c]; k < off[c + 1]; ++k) tab[(size_t)k] = c;
            for (int k = off[n + 1 + c]; k < off[n + 2 + c]; ++k) tab[(size_t)(off[n] + k)] = c;
        }
        BCK(cudaStreamSynchronize(b->stream));
        if (b->item_case_cap < (size_t)items) {
            if (b->d_item_case) cudaFree(b->d_item_case);
            b->d_item_case = nullptr;
            b->item_case_cap = 0;
            BCK(cudaMalloc((void**)&b->d_item_case, sizeof(int) * (size_t)items));
            b->item_case_cap = (size_t)items;
        }
        BCK(cudaMemcpy(b->d_item_case, tab.data(), sizeof(int) * (size_t)items, cudaMemcpyHostToDevice));
        b->item_case_cfg = table_key;
    }

    // the full kernel instantiation when any case has field statistics or a body force in this
    // call, or macroscopic output is asked for; the lean one otherwise
    int full = want_macro ? 1 : 0;
    for (mrlbm_handle* h : b->h) {
        if (h->has_body) full = 1;
        if (h->d_fstat && std::max(h->iter + 1, h->fstat_begin) <= std::min(h->iter + steps, h->fstat_end)) full = 1;
    }
    BatchArgs<double> a64{};
    BatchArgs<float> a32{};
    auto setup = [&](auto& a, auto* params) {
        a.params = params;
        a.cases = b->d_cases;
        a.aux_off = b->d_off;
        a.tile_off = b->d_off + n + 1;
        a.item_case = b->d_item_case;
        a.aux_case = b->d_item_case;                   // split steps: aux items first, then the tiles
        a.tile_case = b->d_item_case + off[n];
        a.bar = b->d_bar;
        a.ncases = n;
        a.call_steps = steps;
        a.want_macro = want_macro;
        a.full = full;
        a.spin_limit = b->wait_limit;
    };
    setup(a64, (const StepParams<double>*)b->d_params);
    setup(a32, (const StepParams<float>*)b->d_params);
    auto launch = [&](int nsteps, int step0, int grid, bool coop) {
        a64.nsteps = a32.nsteps = nsteps;
        a64.step0 = a32.step0 = step0;
        return b->precision == MRLBM_FP64 ? launch_batch_f64(a64, b->tile_cfg, grid, coop, b->stream)
                                          : launch_batch_f32(a32, b->tile_cfg, grid, coop, b->stream);
    };
    // split step k of the call: the auxiliary items walked by two blocks per SM, then the bulk
    // tiles in contiguous runs over eight times the resident blocks (runs short enough that the
    // blocks finish together; measured on the 64-case sweep: 1x 162 us, 4x 143 us, 8x 139 us,
    // 16x 146 us per step)
    const int per_sm_split = batch_split(b) ? batch_split_blocks_per_sm(b->precision, b->tile_cfg) : 0;
    const int split_grid = std::max(1, std::min(off[2 * n + 1], 8 * b->num_sms * std::max(per_sm_split, 1)));
    auto launch_split = [&](int k) {
        a64.nsteps = a32.nsteps = 1;
        a64.step0 = a32.step0 = k;
        const int aux_grid = std::min(off[n], 2 * b->num_sms);
        return b->precision == MRLBM_FP64 ? launch_batch_split_f64(a64, b->tile_cfg, aux_grid, split_grid, b->stream)
                                          : launch_batch_split_f32(a32, b->tile_cfg, aux_grid, split_grid, b->stream);
    };
    if (b->schedule == MRLBM_BATCH_PERSISTENT) {
        const int per_sm = batch_blocks_per_sm(b->precision, b->tile_cfg);
        if (per_sm <= 0) return bfail(b, MRLBM_EUNSUPPORTED, "batch shape does not fit");
        const int grid = std::min(items, b->num_sms * per_sm);
        if (launch(steps, 0, grid, steps > 1) != 0)
            return bfail(b, MRLBM_ECUDA, std::string("batch launch: ") + cudaGetErrorString(cudaGetLastError()));
        ++b->launches;
    } else {
        if (per_sm_split <= 0) return bfail(b, MRLBM_EUNSUPPORTED, "batch shape does not fit");
        if (!b->graph || b->graph_cfg != b->tile_cfg || b->graph_steps != steps || b->graph_macro != want_macro ||
            b->graph_full != full) {
            if (b->graph) cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
            BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            int rc = 0;
            for (int k = 0; k < steps && rc == 0; ++k) rc = launch_split(k);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(b->stream, &g);
            if (rc != 0 || e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                return bfail(b, MRLBM_ECUDA, "capturing the batch step graph failed");
            }
            e = cudaGraphInstantiate(&b->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return bfail(b, MRLBM_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
            b->graph_cfg = b->tile_cfg;
            b->graph_steps = steps;
            b->graph_macro = want_macro;
            b->graph_full = full;
        }
        BCK(cudaGraphLaunch(b->graph, b->stream));
        b->launches += 2 * steps;
    }
    for (mrlbm_handle* h : b->h) {
        const int a0 = h->iter + 1, z = h->iter + steps;
        h->ring_n += stats_in(h->cfg, a0, z);
        if (h->d_fstat) {
            const int lo = std::max(a0, h->fstat_begin), hi = std::min(z, h->fstat_end);
            if (hi >= lo) h->fstat_n += hi - lo + 1;
        }
        h->iter = z;
        h->cur ^= steps & 1;
        h->ovr_live = false;
    }
    return MRLBM_OK;
}

void batch_free(mrlbm_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (auto& q : b->sg)
        if (q.exec) cudaGraphExecDestroy(q.exec);
    for (cudaStream_t s : b->cstream)
        if (s) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->join_ev)
        if (e) cudaEventDestroy(e);
    if (b->fork_ev) cudaEventDestroy(b->fork_ev);
    if (b->call_staged) cudaEventDestroy(b->call_staged);
    if (b->d_call) cudaFree(b->d_call);
    if (b->h_call) cudaFreeHost(b->h_call);
    for (mrlbm_handle* h : b->h) {
        if (!h) continue;
        h->stream = nullptr;
        free_all(h);
        delete h;
    }
    for (void* q : {(void*)b->d_params, (void*)b->d_cases, (void*)b->d_off, (void*)b->d_bar, (void*)b->d_item_case})
        if (q) cudaFree(q);
    for (int i = 0; i < 2; ++i) {
        if (b->h_stage[i]) cudaFreeHost(b->h_stage[i]);
        if (b->staged[i]) cudaEventDestroy(b->staged[i]);
    }
    if (b->stream) cudaStreamDestroy(b->stream);
}

}  // namespace

extern "C" {

int mrlbm_batch_create(const mrlbm_config* cfgs, int32_t ncases, int precision, int device, mrlbm_batch** out) {
    if (!cfgs || !out || ncases <= 0 || device < 0) return MRLBM_EINVAL;
    *out = nullptr;
    mrlbm_batch* b = new mrlbm_batch();
    b->precision = precision;
    b->device = device;
    auto bail = [&](int rc, const std::string& msg) {
        g_create_error = msg;
        batch_free(b);
        delete b;
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(MRLBM_ENODEVICE, "cudaSetDevice failed");
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(MRLBM_ECUDA, "cudaStreamCreate failed");
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
    for (int c = 0; c < ncases; ++c) {
        mrlbm_handle* h = nullptr;
        int rc = mrlbm_create(cfgs + c, precision, device, &h);
        if (rc != MRLBM_OK) return bail(rc, "case " + std::to_string(c) + ": " + g_create_error);
        b->h.push_back(h);
        if (h->own_stream) {
            cudaStreamSynchronize(h->own_stream);
            cudaStreamDestroy(h->own_stream);
            h->own_stream = nullptr;
        }
        h->stream = b->stream;
    }
    b->stage_bytes = batch_param_bytes(b);
    bool ok = cudaMalloc(&b->d_params, b->stage_bytes) == cudaSuccess &&
              cudaMalloc((void**)&b->d_cases, sizeof(BatchCase) * ncases) == cudaSuccess &&
              cudaMalloc((void**)&b->d_off, sizeof(int) * (2 * ncases + 2)) == cudaSuccess &&
              cudaMalloc((void**)&b->d_bar, sizeof(BatchBarrier)) == cudaSuccess &&
              cudaMemsetAsync(b->d_bar, 0, sizeof(BatchBarrier), b->stream) == cudaSuccess;
    for (int i = 0; ok && i < 2; ++i)
        ok = cudaMallocHost((void**)&b->h_stage[i], b->stage_bytes) == cudaSuccess &&
             cudaEventCreateWithFlags(&b->staged[i], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventRecord(b->staged[i], b->stream) == cudaSuccess;
    if (!ok || cudaStreamSynchronize(b->stream) != cudaSuccess) return bail(MRLBM_ECUDA, "batch allocation failed");
    *out = b;
    return MRLBM_OK;
}

int mrlbm_batch_destroy(mrlbm_batch* b) {
    if (!b) return MRLBM_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_free(b);
    delete b;
    return MRLBM_OK;
}

int mrlbm_batch_case(mrlbm_batch* b, int32_t c, mrlbm_handle** h) {
    if (!b || !h || c < 0 || c >= (int)b->h.size()) return MRLBM_EINVAL;
    *h = b->h[c];
    return MRLBM_OK;
}

int mrlbm_batch_set_schedule(mrlbm_batch* b, int32_t tile_cfg, int32_t schedule, int32_t steps_per_launch) {
    // the persistent schedule takes the vector shapes; split steps (graph schedule) also the
    // one-tile-per-block shapes
    const bool tile = tile_cfg >= 0 && tile_cfg < N_TILE_CFGS;
    const bool shape_ok = schedule == MRLBM_BATCH_PERSISTENT ? is_vec_cfg(tile_cfg)
                          : schedule == MRLBM_BATCH_GRAPH     ? is_vec_cfg(tile_cfg) || tile
                          : schedule == MRLBM_BATCH_STREAMS   ? tile
                                                              : false;
    // a per-case streams graph holds cases x steps_per_launch step launches: bounded so that its
    // capture and instantiation stay short
    const int max_spl = schedule == MRLBM_BATCH_STREAMS ? STREAMS_MAX_STEPS : RING_CAP;
    if (!b || !shape_ok || steps_per_launch < 1 || steps_per_launch > max_spl) return MRLBM_EINVAL;
    b->tile_cfg = tile_cfg;
    b->schedule = schedule;
    b->steps_per_launch = steps_per_launch;
    return MRLBM_OK;
}

int mrlbm_batch_set_wait_limit(mrlbm_batch* b, int64_t polls) {
    if (!b || polls < 0 || polls > 0xffffffffLL) return MRLBM_EINVAL;
    b->wait_limit = polls == 0 ? BAR_SPIN_LIMIT : (unsigned)polls;
    return MRLBM_OK;
}

int mrlbm_batch_get_schedule(const mrlbm_batch* b, int32_t* tile_cfg, int32_t* schedule, int32_t* steps_per_launch) {
    if (!b) return MRLBM_EINVAL;
    if (tile_cfg) *tile_cfg = b->tile_cfg;
    if (schedule) *schedule = b->schedule;
    if (steps_per_launch) *steps_per_launch = b->steps_per_launch;
    return MRLBM_OK;
}

int mrlbm_batch_step(mrlbm_batch* b, int32_t nsteps, int32_t flags) {
    if (!b || nsteps < 0) return MRLBM_EINVAL;
    BCK(cudaSetDevice(b->device));
    int done = 0;
    while (done < nsteps) {
        const int s = std::min(b->steps_per_launch, nsteps - done);
        const int rc = batch_call(b, s, (flags & MRLBM_STEP_MACRO) && done + s == nsteps);
        if (rc != MRLBM_OK) return rc;
        done += s;
    }
    return MRLBM_OK;
}

int mrlbm_batch_status(mrlbm_batch* b) {
    if (!b) return MRLBM_EINVAL;
    BCK(cudaSetDevice(b->device));
    BatchBarrier bar{};
    BCK(cudaMemcpyAsync(&bar, b->d_bar, sizeof(bar), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    if (bar.err) return bfail(b, MRLBM_EDEVICE_TIMEOUT, "device flag: batch grid-barrier wait timed out");
    for (size_t c = 0; c < b->h.size(); ++c) {
        const int rc = mrlbm_status(b->h[c]);
        if (rc != MRLBM_OK) return bfail(b, rc, "case " + std::to_string(c) + ": " + b->h[c]->err);
    }
    return MRLBM_OK;
}

int mrlbm_batch_last_error(const mrlbm_batch* b, char* buf, size_t len) {
    if (!buf || len == 0) return MRLBM_EINVAL;
    std::snprintf(buf, len, "%s", b ? b->err.c_str() : g_create_error.c_str());
    return MRLBM_OK;
}

int mrlbm_batch_get_stream(const mrlbm_batch* b, void** stream) {
    if (!b || !stream) return MRLBM_EINVAL;
    *stream = (void*)b->stream;
    return MRLBM_OK;
}

int mrlbm_batch_launch_count(const mrlbm_batch* b, int64_t* n) {
    if (!b || !n) return MRLBM_EINVAL;
    *n = b->launches;
    return MRLBM_OK;
}

int mrlbm_batch_autotune(mrlbm_batch* b, int32_t trial_steps, double* best_ms_per_step) {
    if (!b || trial_steps < 1) return MRLBM_EINVAL;
    BCK(cudaSetDevice(b->device));
    // drain the force rings and save every case's populations, counters and field sums
    struct Saved { void* buf[2]; double* fstat; int iter, cur, ring_n; bool ovr; int64_t fstat_n; size_t hist; };
    std::vector<Saved> sv(b->h.size());
    int rc = MRLBM_OK;
    for (size_t c = 0; c < b->h.size() && rc == MRLBM_OK; ++c) {
        mrlbm_handle* h = b->h[c];
        rc = drain_ring(h);
        if (rc != MRLBM_OK) return bfail(b, rc, h->err);
        Saved& s = sv[c];
        s = Saved{{nullptr, nullptr}, nullptr, h->iter, h->cur, h->ring_n, h->ovr_live, h->fstat_n, h->hist.size()};
        const size_t bytes = (size_t)h->L.total() * h->elem;
        for (int k = 0; k < 2; ++k) {
            BCK(cudaMalloc(&s.buf[k], bytes));
            BCK(cudaMemcpyAsync(s.buf[k], h->buf[k], bytes, cudaMemcpyDeviceToDevice, b->stream));
        }
        if (h->d_fstat) {
            const size_t fb = (size_t)6 * h->L.nx * h->L.ny * sizeof(double);
            BCK(cudaMalloc((void**)&s.fstat, fb));
            BCK(cudaMemcpyAsync(s.fstat, h->d_fstat, fb, cudaMemcpyDeviceToDevice, b->stream));
        }
    }
    auto restore = [&]() {
        for (size_t c = 0; c < b->h.size(); ++c) {
            mrlbm_handle* h = b->h[c];
            Saved& s = sv[c];
            const size_t bytes = (size_t)h->L.total() * h->elem;
            for (int k = 0; k < 2; ++k)
                if (cudaMemcpyAsync(h->buf[k], s.buf[k], bytes, cudaMemcpyDeviceToDevice, b->stream) != cudaSuccess)
                    rc = MRLBM_ECUDA;
            if (s.fstat)
                cudaMemcpyAsync(h->d_fstat, s.fstat, (size_t)6 * h->L.nx * h->L.ny * sizeof(double),
                                cudaMemcpyDeviceToDevice, b->stream);
            h->iter = s.iter;
            h->cur = s.cur;
            h->ring_n = s.ring_n;
            h->ovr_live = s.ovr;
            h->fstat_n = s.fstat_n;
            h->hist.resize(s.hist);
        }
    };
    const int tile0 = b->tile_cfg, sched0 = b->schedule, spl0 = b->steps_per_launch;
    int best_tile = tile0, best_sched = sched0, best_spl = spl0;
    double best = 1e300;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int steps = std::min((trial_steps + 1) & ~1, RING_CAP);   // even: a call ends on its start level
    for (int cfg = 0; cfg < PIPE_CFG0 && rc == MRLBM_OK; ++cfg) {
        if (cfg >= N_TILE_CFGS && cfg < VEC_CFG0) continue;     // TMA shapes are single-case only
        for (int sched = MRLBM_BATCH_PERSISTENT; sched <= MRLBM_BATCH_STREAMS && rc == MRLBM_OK; ++sched) {
            if (!is_vec_cfg(cfg) && sched == MRLBM_BATCH_PERSISTENT) continue;
            if (is_vec_cfg(cfg) && sched == MRLBM_BATCH_STREAMS) continue;
            b->tile_cfg = cfg;
            b->schedule = sched;
            b->steps_per_launch = steps;
            rc = batch_call(b, steps, 0);                    // warm-up (and graph capture)
            if (rc == MRLBM_EUNSUPPORTED) { rc = MRLBM_OK; continue; }
            if (rc != MRLBM_OK) break;
            cudaEventRecord(e0, b->stream);
            rc = batch_call(b, steps, 0);
            cudaEventRecord(e1, b->stream);
            if (rc != MRLBM_OK || cudaEventSynchronize(e1) != cudaSuccess) { rc = rc ? rc : MRLBM_ECUDA; break; }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) { best = ms; best_tile = cfg; best_sched = sched; best_spl = steps; }
            restore();
        }
    }
    restore();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamSynchronize(b->stream);
    for (Saved& s : sv) {
        for (void* q : s.buf) if (q) cudaFree(q);
        if (s.fstat) cudaFree(s.fstat);
    }
    if (rc != MRLBM_OK) {
        b->tile_cfg = tile0; b->schedule = sched0; b->steps_per_launch = spl0;
        return rc;
    }
    b->tile_cfg = best_tile;
    b->schedule = best_sched;
    b->steps_per_launch = best_spl;
    if (best_ms_per_step) *best_ms_per_step = best / steps;
    return MRLBM_OK;
}

}  // extern "C"
