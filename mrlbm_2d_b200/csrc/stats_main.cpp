// stats_main.cpp -- `mrlbm_statistics`: the reference's post-processing program
// (2d_statistics.f90) as a host driver over the public C ABI.  Run it where the reference's
// statistics executable would run, after a run of mrlbm_run (or of the reference itself):
//
//   mrlbm_statistics
//
// Reads (2d_statistics.f90 line of the reader in brackets):
//   input_stat.dat                      &parameters nbct, r_cy, uo, rho_infty        [232-258]
//   data_mean/forces_time.dat           iter, F_drag, F_lift per line (list-directed)  [36-42, 86-90]
//   data_mean/theta.dat                 nbct wall angles in surface order              [80-84]
//   data_mean/p_surface_time.dat,       unformatted records (iter, p by theta)         [100-112]
//   data_mean/p_surface_smooth_time.dat
// Writes:
//   plots/cp.dat, plots/cp_fit.dat      |theta*180/pi - 180|, Cp for theta <= pi        [145-159]
//   plots/cd_time.dat, plots/cl_time.dat  (i - cycle_start)/period (REAL), Cd(i) / Cl(i) [161-170]
//   plots/drag_lift.dat                 St, mean Cd, rms Cl                            [171-175]
// The period, the averages and Cp come from mrlbm_force_statistics / mrlbm_cp_statistics,
// which follow 2d_statistics.f90:90-131 and 183-214 operation by operation.
#include <sys/stat.h>

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mrlbm.h"
#include "fortran_io.h"

namespace {

std::string lower(std::string s) {
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n,"), b = s.find_last_not_of(" \t\r\n,");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// &parameters of input_stat.dat (read_input_file, 2d_statistics.f90:232-258).
bool read_parameters(const char* path, int& nbct, double& r_cy, double& uo, double& rho_infty) {
    std::ifstream in(path);
    if (!in) return false;
    std::stringstream ss;
    ss << in.rdbuf();
    std::string text, raw = ss.str();
    for (size_t a = 0; a < raw.size(); ++a) {                  // drop '!' comments
        if (raw[a] == '!') { while (a < raw.size() && raw[a] != '\n') ++a; }
        if (a < raw.size()) text += raw[a];
    }
    const std::string lt = lower(text);
    size_t g = lt.find("&parameters");
    if (g == std::string::npos) return false;
    size_t e = lt.find('/', g);
    std::string body = text.substr(g + 11, (e == std::string::npos ? text.size() : e) - g - 11);
    for (auto& c : body) if (c == '\n' || c == '\r' || c == '\t') c = ' ';
    bool got[4] = {false, false, false, false};
    size_t p = 0;
    while (true) {
        size_t eq = body.find('=', p);
        if (eq == std::string::npos) break;
        const std::string name = lower(trim(body.substr(p, eq - p)));
        size_t next = body.find('=', eq + 1), vend = body.size();
        if (next != std::string::npos) {
            size_t k = next;
            while (k > eq && body[k - 1] == ' ') --k;
            while (k > eq && body[k - 1] != ' ' && body[k - 1] != ',') --k;
            vend = k;
        }
        std::string val = lower(trim(body.substr(eq + 1, vend - eq - 1)));
        for (auto& c : val) if (c == 'd') c = 'e';
        char* end = nullptr;
        const double x = std::strtod(val.c_str(), &end);
        if (val.empty() || *end != '\0') return false;
        if (name == "nbct") { nbct = (int)x; got[0] = true; }
        else if (name == "r_cy") { r_cy = x; got[1] = true; }
        else if (name == "uo") { uo = x; got[2] = true; }
        else if (name == "rho_infty") { rho_infty = x; got[3] = true; }
        else return false;
        p = vend;
    }
    return got[0] && got[1] && got[2] && got[3];
}

// Unformatted records (iter, p(1..nbct)) of a surface-pressure history; step-major values.
bool read_surface(const char* path, int nstep, int nbct, std::vector<double>& out) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    out.assign((size_t)nstep * nbct, 0.0);
    std::vector<char> r;
    for (int i = 0; i < nstep; ++i) {
        if (!read_fortran_record(f, r) || r.size() < 4 + 8 * (size_t)nbct) { std::fclose(f); return false; }
        std::memcpy(out.data() + (size_t)i * nbct, r.data() + 4, 8 * (size_t)nbct);
    }
    std::fclose(f);
    return true;
}

int fail(const char* msg) {
    std::printf("%s\n", msg);
    return 1;
}

}  // namespace

int main() {
    int nbct = 0;
    double r_cy = 0, uo = 0, rho_infty = 0;
    std::printf(" Reading input_stat.dat file ...\n");
    if (!read_parameters("input_stat.dat", nbct, r_cy, uo, rho_infty) || nbct <= 0)
        return fail("Error while reading input.dat file...");                   // 2d_statistics.f90:244-246
    const double PI = 4.0 * std::atan(1.0);
    // forces_time.dat: one line per stats step (2d_statistics.f90:36-42 count, 86-90 read)
    std::vector<int> it;
    std::vector<double> fd, fl;
    {
        std::ifstream in("data_mean/forces_time.dat");
        if (!in) return fail("cannot open data_mean/forces_time.dat");
        std::string line;
        while (std::getline(in, line)) {
            std::istringstream ls(lower(line));
            std::string a, b, c;
            if (!(ls >> a >> b >> c)) return fail("malformed line in data_mean/forces_time.dat");
            for (std::string* s : {&b, &c}) for (auto& ch : *s) if (ch == 'd') ch = 'e';
            it.push_back(std::atoi(a.c_str()));
            fd.push_back(std::strtod(b.c_str(), nullptr));
            fl.push_back(std::strtod(c.c_str(), nullptr));
        }
    }
    const int nstep = (int)fd.size();
    std::vector<double> theta;
    {
        std::ifstream in("data_mean/theta.dat");
        if (!in) return fail("cannot open data_mean/theta.dat");
        for (int k = 0; k < nbct; ++k) {
            std::string v;
            if (!(in >> v)) return fail("data_mean/theta.dat holds fewer than nbct angles");
            for (auto& ch : v) if (ch == 'd' || ch == 'D') ch = 'e';
            theta.push_back(std::strtod(v.c_str(), nullptr));
        }
    }
    double St = 0, Cd = 0, Cl = 0;
    int32_t cs = 0, per = 0, ncyc = 0;
    int rc = mrlbm_force_statistics(fd.data(), fl.data(), nstep, r_cy, uo, rho_infty, &St, &Cd, &Cl, &cs, &per, &ncyc);
    if (rc == MRLBM_ESTATE) return fail(" Error: Could not detect two peaks.");   // 2d_statistics.f90:205-208
    if (rc != MRLBM_OK) return fail("force statistics failed");
    std::printf(" Averging over %d cycle(s)\n", ncyc);                          // 2d_statistics.f90:93-94
    std::vector<double> ps, psf, cp(nbct), cpf(nbct);
    if (!read_surface("data_mean/p_surface_time.dat", nstep, nbct, ps) ||
        !read_surface("data_mean/p_surface_smooth_time.dat", nstep, nbct, psf))
        return fail("cannot read the surface-pressure histories");
    if (mrlbm_cp_statistics(ps.data(), nstep, nbct, cs, per, ncyc, rho_infty, uo, cp.data()) != MRLBM_OK ||
        mrlbm_cp_statistics(psf.data(), nstep, nbct, cs, per, ncyc, rho_infty, uo, cpf.data()) != MRLBM_OK)
        return fail("surface pressure statistics failed");
    mkdir("plots", 0755);
    const double D_cy = 2.0 * r_cy;
    const double f_norm = 0.50 * rho_infty * (uo * uo) * D_cy;                    // 2d_statistics.f90:32
    const int ce = cs + ncyc * per;
    struct Out { const char* path; const std::vector<double>* v; } cps[2] = {{"plots/cp.dat", &cp}, {"plots/cp_fit.dat", &cpf}};
    for (const Out& o : cps) {
        FILE* f = std::fopen(o.path, "w");
        if (!f) return fail("cannot write plots/");
        for (int k = 0; k < nbct; ++k)
            if (theta[k] <= PI)
                std::fprintf(f, "%s%s\n", ld_real(std::fabs((theta[k] * 180.0 / PI) - 180.0)).c_str(), ld_real((*o.v)[k]).c_str());
        std::fclose(f);
    }
    const double* sig[2] = {fd.data(), fl.data()};
    const char* tpath[2] = {"plots/cd_time.dat", "plots/cl_time.dat"};
    for (int q = 0; q < 2; ++q) {
        FILE* f = std::fopen(tpath[q], "w");
        if (!f) return fail("cannot write plots/");
        for (int i = cs; i <= ce; ++i) {
            const float phase = (float)(i - cs) / (float)per;                     // REAL division
            std::fprintf(f, "%s%s\n", ld_real4(phase).c_str(), ld_real(sig[q][i - 1] / f_norm).c_str());
        }
        std::fclose(f);
    }
    const char* labels[3] = {"Strouhal number (St)  ", "Drag coefficinet (C_D)  ", "Lift coefficinet (C_L "};
    const double vals[3] = {St, Cd, Cl};
    FILE* f = std::fopen("plots/drag_lift.dat", "w");
    if (!f) return fail("cannot write plots/");
    for (int q = 0; q < 3; ++q) {
        std::fprintf(f, " %s:%s\n", labels[q], ld_real(vals[q]).c_str());
        std::printf(" %s:%s\n", labels[q], ld_real(vals[q]).c_str());
    }
    std::fclose(f);
    return 0;
}
