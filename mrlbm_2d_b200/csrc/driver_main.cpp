// driver_main.cpp -- `mrlbm_run`: the reference's main program (2d_mrlbm.f90:77-555) as a
// host driver over the public C ABI.  Run it where the reference's a.out would run: it reads
// ./input.dat and writes the reference's output files in their formats.
//
//   mrlbm_run [--fp32] [--device N] [--print-every N]
//
// Files (2d_mrlbm.f90 line of the writer in brackets):
//   output/grid.x                       PLOT3D grid, Fortran unformatted          [2133-2160]
//   output/gridNNNNNNNN.bin             PLOT3D function (rho, ux, uy as float32)   [2163-2184]
//   output/master.p3d                   index of the function files                [2334-2367]
//   restart/restart.dat                 soln_time, f, f_eq, ux, uy, rho            [2186-2202]
//   data_mean/forces_time.dat           iter, F_drag_net, F_lift_net per stats step [492-494]
//   data_mean/p_surface_time.dat,       unformatted records (iter, wall pressure by theta) and
//   data_mean/p_surface_smooth_time.dat its Gaussian smoothing, per stats step          [593-616]
//   data_probe/{p,ux,uy}_probe.dat      iter and the 4 probes' rho/3, ux/3, uy/3        [462-476]
//   data_mean/theta.dat                 sorted wall angles                         [1158-1162]
//   rho_mean_inlet.dat                  running mean inlet density /100 stats steps [362-366]
//   data_probe/probe_loc.dat, simulation_parameters.dat                            [113-118, 157-168]
// Stdout: the STEP / MAX_ux / MLUPS line every 100 steps (MLUPS here is wall-clock).
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mrlbm.h"
#include "fortran_io.h"

namespace {

void die(const char* what, int rc, mrlbm_handle* h) {
    char buf[1024] = {0};
    mrlbm_last_error(h, buf, sizeof buf);
    std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, buf);
    std::exit(1);
}

void mkdirs() {
    for (const char* d : {"output", "restart", "data_probe", "data_geo", "data_mean"}) mkdir(d, 0755);
}

}  // namespace

int main(int argc, char** argv) {
    int precision = MRLBM_FP64, device = 0, print_every = 100;
    for (int a = 1; a < argc; ++a) {
        if (!std::strcmp(argv[a], "--fp32")) precision = MRLBM_FP32;
        else if (!std::strcmp(argv[a], "--device") && a + 1 < argc) device = std::atoi(argv[++a]);
        else if (!std::strcmp(argv[a], "--print-every") && a + 1 < argc) print_every = std::atoi(argv[++a]);
    }
    mrlbm_config cfg;
    mrlbm_config_defaults(&cfg);
    std::printf(" Reading input.dat file ...\n");
    int rc = mrlbm_config_from_namelist("input.dat", &cfg);
    if (rc != MRLBM_OK) {
        std::printf("Error while reading input.dat file...\n");     // 2d_mrlbm.f90:2235-2237
        return 1;
    }
    mrlbm_config_resolve_geometry(&cfg);
    std::printf("                Reynolds number (Re) is      %15.5g\n", cfg.Re);
    mkdirs();
    mrlbm_handle* h = nullptr;
    if ((rc = mrlbm_create(&cfg, precision, device, &h)) != MRLBM_OK) die("mrlbm_create", rc, nullptr);
    mrlbm_geometry_info gi;
    mrlbm_get_geometry_info(h, &gi);
    const int nx = gi.nx, ny = gi.ny, nb = gi.nbct;
    const size_t N = (size_t)nx * ny;

    {   // PLOT3D grid (2d_mrlbm.f90:2133-2160): coordinates (i-1, j-1) as float32
        FortranWriter w("output/grid.x");
        w.put1<int32_t>(1);
        w.end_record();
        w.put1<int32_t>(nx);
        w.put1<int32_t>(ny);
        w.end_record();
        std::vector<float> xy(2 * N);
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                xy[(size_t)j * nx + i] = (float)i;
                xy[N + (size_t)j * nx + i] = (float)j;
            }
        w.put(xy.data(), xy.size());
        w.end_record();
    }
    // probes on the wake centreline (2d_mrlbm.f90:104-118)
    const int nfront = cfg.L_front * cfg.ncy, nbot = cfg.L_bot * cfg.ncy, ncy = cfg.ncy;
    const int pi_[4] = {(nfront + ncy + 1) + (ncy / 2), (nfront + ncy + 1) + ncy, (nfront + ncy + 1) + (3 * ncy / 2),
                        (nfront + ncy + 1) + (2 * ncy)};
    const int pj = nbot + (ncy / 2) + 1;
    if (FILE* f = std::fopen("data_probe/probe_loc.dat", "w")) {
        for (int q = 0; q < 4; ++q) std::fprintf(f, " probe %d: %s%s\n", q + 1, ld_int(pi_[q]).c_str(), ld_int(pj).c_str());
        std::fclose(f);
    }
    // master.p3d (2d_mrlbm.f90:2334-2367)
    const double L_lat = 2.0 * gi.r_cyl, nu_phy = 0.01, L_phy = 1.0;
    const double delx_phy = L_phy / L_lat, delt_phy = (delx_phy * delx_phy) * gi.nu / nu_phy;
    if (FILE* f = std::fopen("output/master.p3d", "w")) {
        std::fprintf(f, " {\n\n \"auto-detect-format\" : true,\n\n \"filenames\" : [\n\n");
        for (long long it = 0; it <= 10000LL * cfg.iplot; it += std::max(cfg.iplot, 1))
            std::fprintf(f, " { \"time\" :%s,\"xyz\" : \"grid.x\", \"function\" : \"grid%08lld.bin\" },\n",
                         ld_real(it * delt_phy).c_str(), 10000000LL + it);
        std::fprintf(f, "\n ]\n }\n");
        std::fclose(f);
    }
    if (FILE* f = std::fopen("simulation_parameters.dat", "w")) {          // 2d_mrlbm.f90:157-168
        std::fprintf(f, " nx,ny%s%s\n", ld_int(nx).c_str(), ld_int(ny).c_str());
        std::fprintf(f, " No. of points on diameter%s\n", ld_int(ncy).c_str());
        std::fprintf(f, " centre_cylin%s%s\n", ld_int(nfront + ncy / 2).c_str(), ld_int(nbot + ncy / 2 - 1).c_str());
        std::fprintf(f, " Maximum_radius%s\n", ld_real(gi.r_cyl).c_str());
        std::fprintf(f, " No. of points on cylinder:%s\n", ld_int(nb).c_str());
        std::fprintf(f, " Re:%s\n uo:%s\n nu:%s\n tau:%s\n dt_phy:%s\n", ld_real(cfg.Re).c_str(), ld_real(cfg.uo).c_str(),
                     ld_real(gi.nu).c_str(), ld_real(1.0 / gi.omega).c_str(), ld_real(delt_phy).c_str());
        std::fclose(f);
    }
    // theta.dat: wall angles sorted by the reference's selection swap (2d_mrlbm.f90:1132-1162)
    if (nb > 0) {
        std::vector<double> ref(8 * (size_t)nb), th(nb);
        mrlbm_get_boundary_nodes(h, nullptr, nullptr, nullptr, nullptr, ref.data(), nullptr);
        const double PI = 4.0 * std::atan(1.0);
        for (int l = 0; l < nb; ++l) {
            double t = std::atan2(ref[8 * (size_t)l + 4] - gi.y_c, ref[8 * (size_t)l] - gi.x_c);
            if (t < 0) t = t + 2.0 * PI;
            th[l] = t;
        }
        std::vector<int> idx(nb);
        for (int i = 0; i < nb; ++i) idx[i] = i;
        for (int i = 0; i < nb - 1; ++i)
            for (int j = i + 1; j < nb; ++j)
                if (th[idx[i]] > th[idx[j]]) std::swap(idx[i], idx[j]);
        if (FILE* f = std::fopen("data_mean/theta.dat", "w")) {
            for (int i = 0; i < nb; ++i) std::fprintf(f, "%s\n", ld_real(th[idx[i]]).c_str());
            std::fclose(f);
        }
    }
    std::vector<double> rho(N), ux(N), uy(N), fbuf(N * 9);
    auto write_function = [&](long long it) {          // 2d_mrlbm.f90:2163-2184
        char name[64];
        std::snprintf(name, sizeof name, "output/grid%08lld.bin", 10000000LL + it);
        FortranWriter w(name);
        w.put1<int32_t>(1);
        w.end_record();
        w.put1<int32_t>(nx); w.put1<int32_t>(ny); w.put1<int32_t>(3);
        w.end_record();
        std::vector<float> v(3 * N);
        for (size_t n = 0; n < N; ++n) { v[n] = (float)rho[n]; v[N + n] = (float)ux[n]; v[2 * N + n] = (float)uy[n]; }
        w.put(v.data(), v.size());
        w.end_record();
    };
    int iter = 1;
    if (cfg.irestart == 0) {
        std::fill(rho.begin(), rho.end(), 1.0);            // 2d_mrlbm.f90:199-206
        std::fill(ux.begin(), ux.end(), 0.0);
        std::fill(uy.begin(), uy.end(), 0.0);
        write_function(0);
        mrlbm_get_iter(h, &iter);
    } else {                                               // 2d_mrlbm.f90:208-212, 2204-2220
        FILE* f = std::fopen("restart/restart.dat", "rb");
        std::vector<char> r;
        if (!f || !read_fortran_record(f, r) || r.size() < 4 + 8 * (N * 9)) {
            std::fprintf(stderr, "cannot read restart/restart.dat\n");
            return 1;
        }
        std::fclose(f);
        int32_t soln;
        std::memcpy(&soln, r.data(), 4);
        std::memcpy(fbuf.data(), r.data() + 4, 8 * N * 9);
        iter = soln;
        if ((rc = mrlbm_load_state(h, fbuf.data(), soln)) != MRLBM_OK) die("mrlbm_load_state", rc, h);
        std::printf(" Restarting step = %s\n", ld_int(iter).c_str());
    }
    for (const char* p : {"data_mean/p_surface_time.dat", "data_mean/p_surface_smooth_time.dat",
                          "data_mean/forces_time.dat", "rho_mean_inlet.dat"})
        if (FILE* f = std::fopen(p, "w")) std::fclose(f);
    const bool pp = cfg.post_process != 0;
    const int nbct = gi.nbct;
    // surface pressure and probe records of every statistics step (2d_mrlbm.f90:462-476, 593-616)
    const bool surf = pp && nbct > 0 && mrlbm_surface_enable(h, 1) == MRLBM_OK;
    // the reference opens the probe files when iter == statsbegin; a run that starts later
    // writes to the units' default files
    const bool probes_named = cfg.statsbegin > iter;
    const char* probe_file[3] = {probes_named ? "data_probe/p_probe.dat" : "fort.101",
                                 probes_named ? "data_probe/ux_probe.dat" : "fort.102",
                                 probes_named ? "data_probe/uy_probe.dat" : "fort.103"};
    if (surf)
        for (const char* pf : probe_file)
            if (FILE* f = std::fopen(pf, "w")) std::fclose(f);
    std::vector<int32_t> sit(1024);
    std::vector<double> sps((size_t)1024 * std::max(nbct, 1)), spf((size_t)1024 * std::max(nbct, 1)), spr(1024 * 12);
    auto drain_surface = [&]() {
        if (!surf) return;
        int32_t n = 0;
        do {
            if ((rc = mrlbm_get_surface(h, sit.data(), sps.data(), spf.data(), spr.data(), 1024, &n)) != MRLBM_OK)
                die("mrlbm_get_surface", rc, h);
            FortranWriter ws("data_mean/p_surface_time.dat", "ab"), wf("data_mean/p_surface_smooth_time.dat", "ab");
            FILE* fp[3];
            for (int q = 0; q < 3; ++q) fp[q] = std::fopen(probe_file[q], "a");
            for (int t = 0; t < n; ++t) {
                ws.put1(sit[t]);
                ws.put(sps.data() + (size_t)t * nbct, nbct);
                ws.end_record();
                wf.put1(sit[t]);
                wf.put(spf.data() + (size_t)t * nbct, nbct);
                wf.end_record();
                for (int q = 0; q < 3; ++q) {
                    if (!fp[q]) continue;
                    std::fprintf(fp[q], "%s", ld_int(sit[t]).c_str());
                    for (int k = 0; k < 4; ++k) std::fprintf(fp[q], "%s", ld_real(spr[(size_t)t * 12 + 4 * q + k]).c_str());
                    std::fprintf(fp[q], "\n");
                }
            }
            for (int q = 0; q < 3; ++q) if (fp[q]) std::fclose(fp[q]);
        } while (n == 1024);
    };
    double rho_inf_mean = 0.0;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<int32_t> rit(8192);
    std::vector<double> rfd(8192), rfl(8192), rin(8192);
    auto drain = [&]() {
        int32_t n = 0;
        do {
            if ((rc = mrlbm_get_forces(h, rit.data(), rfd.data(), rfl.data(), rin.data(), 8192, &n)) != MRLBM_OK)
                die("mrlbm_get_forces", rc, h);
            FILE* ff = std::fopen("data_mean/forces_time.dat", "a");
            FILE* fr = nullptr;
            for (int t = 0; t < n; ++t) {
                std::fprintf(ff, "%s%s%s\n", ld_int(rit[t]).c_str(), ld_real(rfd[t]).c_str(), ld_real(rfl[t]).c_str());
                const double c = (double)(float)(rit[t] - cfg.statsbegin);   // 2d_mrlbm.f90:358-360
                const double rinf = rin[t] / (double)ny;
                rho_inf_mean = ((c * rho_inf_mean) + rinf) / (c + 1.0);
                if (rit[t] % 100 == 0) {
                    if (!fr) fr = std::fopen("rho_mean_inlet.dat", "a");
                    std::fprintf(fr, "%s%s\n", ld_int(rit[t]).c_str(), ld_real(rho_inf_mean).c_str());
                }
            }
            std::fclose(ff);
            if (fr) std::fclose(fr);
        } while (n == 8192);
        drain_surface();
    };
    const int iplot = std::max(cfg.iplot, 1), isave = std::max(cfg.isave, 1);
    while (iter < cfg.max_iter) {
        // run to the next step that needs the host: output, restart, progress line
        auto next_mult = [&](int m) { return ((iter / m) + 1) * m; };
        int target = cfg.max_iter;
        if (pp) target = std::min(target, next_mult(iplot));
        target = std::min(target, next_mult(isave));
        target = std::min(target, next_mult(print_every));
        if ((rc = mrlbm_step(h, target - iter, MRLBM_STEP_MACRO)) != MRLBM_OK) die("mrlbm_step", rc, h);
        iter = target;
        if ((rc = mrlbm_get_macro(h, rho.data(), ux.data(), uy.data(), nullptr, nullptr, nullptr)) != MRLBM_OK)
            die("mrlbm_get_macro", rc, h);
        if (pp) drain();
        if (pp && iter % iplot == 0) write_function(iter);
        if (iter % print_every == 0) {
            auto t1 = std::chrono::steady_clock::now();
            const double el = std::chrono::duration<double>(t1 - t0).count();
            t0 = t1;
            const double mlups = (double)N * print_every / (1.0e6 * el);
            std::printf(" STEP: %s      MAX_ux: %14.7g      MLUPS: %14.7g\n", ld_int(iter).c_str(),
                        (float)*std::max_element(ux.begin(), ux.end()), (float)mlups);
            std::fflush(stdout);
            if ((rc = mrlbm_status(h)) != MRLBM_OK) die("mrlbm_status", rc, h);
        }
        if (iter % isave == 0) {                           // 2d_mrlbm.f90:550-552, 2186-2202
            std::printf(" Writing restart file at%s iteration\n", ld_int(iter).c_str());
            if ((rc = mrlbm_get_state(h, fbuf.data())) != MRLBM_OK) die("mrlbm_get_state", rc, h);
            FortranWriter w("restart/restart.dat");
            w.put1<int32_t>(iter);
            w.put(fbuf.data(), fbuf.size());
            std::vector<double> feq(N * 9, 0.0);         // f_eq is never set by the reference
            w.put(feq.data(), feq.size());
            w.put(ux.data(), N);
            w.put(uy.data(), N);
            w.put(rho.data(), N);
            w.end_record();
        }
    }
    mrlbm_destroy(h);
    return 0;
}
