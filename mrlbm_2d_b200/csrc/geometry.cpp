// geometry.cpp -- one-off FP64 setup on the host: lattice tables, curved-wall geometry,
// namelist input, initial state.  Compiled with -ffp-contract=off so every value matches
// the reference's FP64 arithmetic bit for bit.
#include "geometry.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

namespace mrlbm {

Lattice64 make_lattice() {
    Lattice64 L;
    const float w0 = 16.0f / 36.0f, w1 = 4.0f / 36.0f, w5 = 1.0f / 36.0f;   // 2d_mrlbm.f90:129
    const double wl[Q] = {w0, w1, w1, w1, w1, w5, w5, w5, w5};
    L.cs2 = 1.0 / 3.0;                                                      // 2d_mrlbm.f90:153
    for (int k = 0; k < Q; ++k) {                                           // 2d_mrlbm.f90:171-174
        L.w[k] = wl[k];
        L.hxx[k] = (double)(ex(k) * ex(k)) - L.cs2;
        L.hyy[k] = (double)(ey(k) * ey(k)) - L.cs2;
        L.hxy[k] = (double)(ex(k) * ey(k));
    }
    L.hm = 0.0 - L.cs2;
    L.hp = 1.0 - L.cs2;
    return L;
}

void link_tables(int label15_rule, int incs[16], int outs[16]) {
    // Rows of Incs_b / Outs_b (2d_mrlbm.f90:2011-2057) as bit masks, bit k = population k.
    auto bits = [](const char* s) { int m = 0; for (int k = 0; k < Q; ++k) if (s[k] == '1') m |= 1 << k; return m; };
    for (int l = 0; l < 16; ++l) { incs[l] = 0; outs[l] = 0; }
    incs[1] = bits("110010001");  outs[1] = bits("101100100");
    incs[2] = bits("100110010");  outs[2] = bits("111001000");
    incs[3] = bits("110110011");  outs[3] = bits("111101100");
    incs[4] = bits("111001000");  outs[4] = bits("100110010");
    incs[5] = bits("111011001");  outs[5] = bits("101110110");
    incs[7] = bits("111111011");  outs[7] = bits("111111110");
    incs[8] = bits("101100100");  outs[8] = bits("110010001");
    incs[10] = bits("101110110"); outs[10] = bits("111011001");
    incs[11] = bits("111110111"); outs[11] = bits("111111101");
    incs[12] = bits("111101100"); outs[12] = bits("110110011");
    incs[13] = bits("111111101"); outs[13] = bits("111110111");
    incs[14] = bits("111111110"); outs[14] = bits("111111011");
    if (label15_rule == MRLBM_LABEL15_ALLNINE) { incs[15] = 0x1ff; outs[15] = 0x1ff; }
}

void resolve_domain(const mrlbm_config& c, int& nx, int& ny, double& x_c, double& y_c, double& r_c) {
    if (c.geometry_mode == MRLBM_GEOM_REFERENCE && c.channel_with_cylinder) {
        const int nfront = c.L_front * c.ncy, nback = c.L_back * c.ncy;
        const int ntop = c.L_top * c.ncy, nbot = c.L_bot * c.ncy;
        nx = nfront + c.ncy + nback;                                         // 2d_mrlbm.f90:91-92
        ny = ntop + c.ncy + nbot;
        x_c = (double)(float)(nfront + (c.ncy / 2) + 1);                     // real(): default kind
        y_c = (double)(float)(nbot + c.ncy / 2);
        r_c = (double)(float)(c.ncy / 2);
    } else {
        nx = c.nx; ny = c.ny; x_c = c.x_c; y_c = c.y_c; r_c = c.r_c;
    }
}

int build_geometry(const mrlbm_config& cfg, int nx, int ny, double x_c, double y_c, double r_c,
                   Geometry& g, std::string& err) {
    g = Geometry();
    g.nx = nx; g.ny = ny; g.x_c = x_c; g.y_c = y_c; g.r_c = r_c;
    g.cylinder = cfg.channel_with_cylinder != 0;
    const size_t N = (size_t)nx * ny;
    g.cls.assign(N, 0);
    if (!g.cylinder) return MRLBM_OK;
    auto id = [nx](int i, int j) { return (size_t)(i - 1) + (size_t)nx * (size_t)(j - 1); };
    auto dist = [&](int i, int j) {
        const double dx = (double)i - x_c, dy = (double)j - y_c;
        return std::sqrt(dx * dx + dy * dy);
    };
    // classification, 2d_mrlbm.f90:969-980 (epsilon is the single-precision 0.5)
    std::vector<int8_t>& cl = g.cls;
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j) {
            const double d = dist(i, j);
            cl[id(i, j)] = std::fabs(d - r_c) <= 0.5 ? 2 : (std::fabs(d) <= r_c ? 1 : 0);
        }
    // every non-fluid 8-neighbour of an interior fluid node becomes a boundary node
    // (2d_mrlbm.f90:982-1002); fluid nodes never change, so the order is immaterial
    std::vector<int8_t> fluid(N);
    for (size_t o = 0; o < N; ++o) fluid[o] = cl[o] == 0;
    for (int i = 2; i <= nx - 1; ++i)
        for (int j = 2; j <= ny - 1; ++j) {
            if (!fluid[id(i, j)]) continue;
            for (int di = -1; di <= 1; ++di)
                for (int dj = -1; dj <= 1; ++dj)
                    if (cl[id(i + di, j + dj)] == 1) cl[id(i + di, j + dj)] = 2;
        }
    // boundary list in (i-major, j-minor) order and quadrant labels, 2d_mrlbm.f90:1007-1036
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j) {
            if (cl[id(i, j)] != 2) continue;
            if (i < 2 || i > nx - 1 || j < 2 || j > ny - 1) {
                err = "curved-wall boundary node on the domain edge";
                return MRLBM_EGEOMETRY;
            }
            auto F = [&](int a, int b) { return fluid[id(a, b)] ? 1 : 0; };
            const int q0 = (F(i - 1, j) | F(i - 1, j + 1) | F(i, j + 1));
            const int q1 = (F(i + 1, j) | F(i + 1, j + 1) | F(i, j + 1));
            const int q2 = (F(i - 1, j) | F(i - 1, j - 1) | F(i, j - 1));
            const int q3 = (F(i + 1, j) | F(i + 1, j - 1) | F(i, j - 1));
            g.bi.push_back(i);
            g.bj.push_back(j);
            g.label.push_back(q0 + 2 * q1 + 4 * q2 + 8 * q3);
        }
    const int nb = (int)g.bi.size();
    g.nb = nb;
    int incs[16], outs[16];
    link_tables(cfg.label15_rule, incs, outs);
    for (int l = 0; l < nb; ++l) {
        if (g.label[l] == 15) ++g.n_label15;
        if (incs[g.label[l]] == 0 && outs[g.label[l]] == 0) {
            char b[200];
            std::snprintf(b, sizeof b,
                          "boundary node %d at (%d,%d) has quadrant label %d, whose link rows are empty "
                          "in the reference (2d_mrlbm.f90:2008); label15_rule=ALLNINE closes label 15",
                          l + 1, g.bi[l], g.bj[l], g.label[l]);
            err = b;
            return MRLBM_EGEOMETRY;
        }
    }
    // r_cyl = largest boundary-node radius, 2d_mrlbm.f90:1038-1050
    double rmax = nb ? dist(g.bi[0], g.bj[0]) : 0.0;
    for (int l = 1; l < nb; ++l) rmax = std::max(rmax, dist(g.bi[l], g.bj[l]));
    g.r_cyl = rmax;

    // wall point, reference points, delta and stencils, 2d_mrlbm.f90:1055-1135
    const double delx = std::sqrt(2.0);
    const double PI = 4.0 * std::atan(1.0);
    g.delta.resize(nb); g.ref.resize(8 * (size_t)nb); g.sten.resize(24 * (size_t)nb); g.theta.resize(nb);
    g.tint.assign((size_t)I_NFIELDS * nb, 0);
    g.tgeo.assign((size_t)G_NFIELDS * nb, 0.0);
    const Lattice64 lat = make_lattice();
    auto rot = [&](int i, int j, double& c, double& s, double& s2, double& c2) {   // 2d_mrlbm.f90:958-966
        const double radi = std::sqrt((((double)i - x_c) * ((double)i - x_c)) + (((double)j - y_c) * ((double)j - y_c)));
        c = ((double)i - x_c) / radi;
        s = ((double)j - y_c) / radi;
        s2 = 2.0 * s * c;
        c2 = (c * c) - (s * s);
    };
    auto T = [&](int field, int l) -> double& { return g.tgeo[(size_t)field * nb + l]; };
    auto TI = [&](int field, int l) -> int& { return g.tint[(size_t)field * nb + l]; };
    for (int l = 0; l < nb; ++l) {
        const int i = g.bi[l], j = g.bj[l];
        const double rr = dist(i, j);
        double unx, uny, xb, yb;
        if (rr > 1.0e-12) {
            unx = ((double)i - x_c) / rr;
            uny = ((double)j - y_c) / rr;
            xb = x_c + (g.r_cyl * unx);
            yb = y_c + (g.r_cyl * uny);
        } else {
            unx = 0.0; uny = 0.0; xb = x_c; yb = y_c;
        }
        double xr[4], yr[4];
        xr[0] = xb;                         yr[0] = yb;
        xr[1] = xb + (delx * unx);          yr[1] = yb + (delx * uny);
        xr[2] = xb + (2.0 * delx * unx);    yr[2] = yb + (2.0 * delx * uny);
        xr[3] = xb + (3.0 * delx * unx);    yr[3] = yb + (3.0 * delx * uny);
        for (int r = 0; r < 4; ++r) { g.ref[8 * (size_t)l + r] = xr[r]; g.ref[8 * (size_t)l + 4 + r] = yr[r]; }
        const double ddx = (double)i - xb, ddy = (double)j - yb;
        const double d = std::sqrt(ddx * ddx + ddy * ddy);
        g.delta[l] = d;
        double th = std::atan2(yb - y_c, xb - x_c);
        if (th < 0) th = th + 2.0 * PI;
        g.theta[l] = th;
        // stencils of reference points 2, 3, 4: corners (fx,fy) (fx+1,fy) (fx,fy+1) (fx+1,fy+1)
        for (int r = 1; r <= 3; ++r) {
            const int fx = (int)std::floor(xr[r]), fy = (int)std::floor(yr[r]);
            const int ci[4] = {fx, fx + 1, fx, fx + 1}, cj[4] = {fy, fy, fy + 1, fy + 1};
            for (int c = 0; c < 4; ++c) {
                const int si = ci[c], sj = cj[c];
                if (si < 2 || si > nx - 1 || sj < 2 || sj > ny - 1 || cl[id(si, sj)] != 0) {
                    char b[200];
                    std::snprintf(b, sizeof b, "stencil node (%d,%d) of boundary node %d is not an interior fluid node",
                                  si, sj, l + 1);
                    err = b;
                    return MRLBM_EGEOMETRY;
                }
                g.sten[24 * (size_t)l + 8 * (r - 1) + c] = si;
                g.sten[24 * (size_t)l + 8 * (r - 1) + 4 + c] = sj;
                TI(I_SI + 4 * (r - 1) + c, l) = si;
                TI(I_SJ + 4 * (r - 1) + c, l) = sj;
                if (r <= 2) {
                    double c0, s0, s20, c20;
                    rot(si, sj, c0, s0, s20, c20);
                    const int m = 4 * (r - 1) + c;
                    T(G_SCC + m, l) = c0 * c0;
                    T(G_SSS + m, l) = s0 * s0;
                    T(G_SS2 + m, l) = s20;
                }
            }
            T(G_XD2 + 2 * (r - 1), l) = (xr[r] - (double)fx) / 1.0;
            T(G_YD2 + 2 * (r - 1), l) = (yr[r] - (double)fy) / 1.0;
        }
        // own-node rotation and rotated lattice (2d_mrlbm.f90:183-197)
        double c, s, s2, c2;
        rot(i, j, c, s, s2, c2);
        T(G_CTH, l) = c; T(G_STH, l) = s; T(G_S2TH, l) = s2; T(G_C2TH, l) = c2;
        T(G_CC, l) = c * c; T(G_SS, l) = s * s;
        for (int k = 0; k < Q; ++k) {
            const double e1 = (double)ex(k), e2 = (double)ey(k);
            T(G_CXP + k, l) = e1 * c + e2 * s;
            T(G_CYP + k, l) = -(e1 * s) + e2 * c;
            T(G_HXXP + k, l) = lat.hxx[k] * (c * c) + lat.hyy[k] * (s * s) + lat.hxy[k] * s2;
            T(G_HYYP + k, l) = lat.hxx[k] * (s * s) + lat.hyy[k] * (c * c) - lat.hxy[k] * s2;
            T(G_HXYP + k, l) = (lat.hyy[k] - lat.hxx[k]) * 0.50 * s2 + lat.hxy[k] * c2;
        }
        // quadratic extrapolation weights (2d_mrlbm.f90:809-811)
        T(G_T1, l) = (2.0 * delx * delx - (d * d) + 3.0 * d * delx) / (2.0 * (delx * delx));
        T(G_T2, l) = d * (d - 2.0 * delx) / (delx * delx);
        T(G_T3, l) = d * (d - delx) / (2.0 * (delx * delx));
        TI(I_NODEI, l) = i;
        TI(I_NODEJ, l) = j;
        TI(I_IS, l) = incs[g.label[l]];
        TI(I_OS, l) = outs[g.label[l]];
        TI(I_LABEL, l) = g.label[l];
    }
    // bounding box of every non-fluid node; edge rows/columns must stay fluid
    int x0 = nx + 1, x1 = 0, y0 = ny + 1, y1 = 0;
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j)
            if (cl[id(i, j)] != 0) {
                if (i == 1 || i == nx || j == 1 || j == ny) {
                    err = "the cylinder touches the domain edge";
                    return MRLBM_EGEOMETRY;
                }
                x0 = std::min(x0, i); x1 = std::max(x1, i); y0 = std::min(y0, j); y1 = std::max(y1, j);
            }
    if (x1 >= x0) {
        g.box_x0 = x0; g.box_y0 = y0; g.box_w = x1 - x0 + 1; g.box_h = y1 - y0 + 1;
        g.boxmap.assign((size_t)g.box_w * g.box_h, CLS_FLUID);
        for (int i = x0; i <= x1; ++i)
            for (int j = y0; j <= y1; ++j)
                if (cl[id(i, j)] == 1) g.boxmap[(size_t)(j - y0) * g.box_w + (i - x0)] = CLS_SOLID;
        for (int l = 0; l < nb; ++l) g.boxmap[(size_t)(g.bj[l] - y0) * g.box_w + (g.bi[l] - x0)] = l;
    }
    return MRLBM_OK;
}

// ---------------------------------------------------------------------------------------
void config_defaults(mrlbm_config& c) {
    std::memset(&c, 0, sizeof c);
    c.nx = 320; c.ny = 32; c.lattice_type = 9;                   // input.dat:1-5
    c.ncy = 20; c.L_front = 10; c.L_back = 35; c.L_top = 10; c.L_bot = 10;
    c.Re = 100.0;
    c.num_threads = 16;
    c.uo = 0.1; c.rho_infty = 1.0; c.iplot = 100; c.max_iter = 900000000; c.isave = 10000;
    c.irestart = 0; c.statsbegin = 100001; c.statsend = 200001; c.iplotstats = 1000;
    c.post_process = 1; c.x_periodic = 0; c.y_periodic = 1; c.channel_with_cylinder = 1;
    c.channel_with_square = 0; c.incomp_bc = 0; c.incomp_bulk = 0; c.vel_interp = 1; c.mom_interp = 1;
    c.rotated_coordinate = 1; c.strong_mass_bc = 1; c.eq_mass_bc = 0; c.weak_mass_bc = 0;
    c.noise_amp = 1e-4; c.seed = 0;
}

namespace {
std::string lower(std::string s) { for (auto& ch : s) ch = (char)std::tolower((unsigned char)ch); return s; }
std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}
bool parse_logical(const std::string& v, int& out) {
    std::string t = lower(trim(v));
    if (!t.empty() && t[0] == '.') t = t.substr(1);
    if (t.empty()) return false;
    if (t[0] == 't') { out = 1; return true; }
    if (t[0] == 'f') { out = 0; return true; }
    return false;
}
bool parse_int(const std::string& v, int& out) {
    std::string t = trim(v);
    if (t.empty()) return false;
    char* end = nullptr;
    long x = std::strtol(t.c_str(), &end, 10);
    if (*end != '\0') return false;
    out = (int)x;
    return true;
}
bool parse_real(const std::string& v, double& out) {
    std::string t = lower(trim(v));
    for (auto& ch : t) if (ch == 'd' || ch == 'q') ch = 'e';     // Fortran exponent letters
    if (t.empty()) return false;
    char* end = nullptr;
    double x = std::strtod(t.c_str(), &end);
    if (*end != '\0') return false;
    out = x;
    return true;
}
}  // namespace

int read_namelist_file(const char* path, mrlbm_config& cfg, std::string& err) {
    std::ifstream in(path);
    if (!in) { err = std::string("cannot open ") + path; return MRLBM_ENAMELIST; }
    std::stringstream ss;
    ss << in.rdbuf();
    std::string text = ss.str();
    // strip comments ('!' outside quotes) and split into groups &name ... /
    std::string clean;
    bool inq = false;
    for (size_t a = 0; a < text.size(); ++a) {
        char ch = text[a];
        if (ch == '\'' || ch == '"') inq = !inq;
        if (ch == '!' && !inq) { while (a < text.size() && text[a] != '\n') ++a; clean += '\n'; continue; }
        clean += ch;
    }
    std::map<std::string, std::string> groups;
    std::vector<std::string> order;
    size_t pos = 0;
    while ((pos = clean.find('&', pos)) != std::string::npos) {
        size_t ne = clean.find_first_of(" \t\r\n", pos);
        if (ne == std::string::npos) break;
        std::string name = lower(clean.substr(pos + 1, ne - pos - 1));
        size_t endg = clean.find('/', ne);
        if (endg == std::string::npos) { err = "namelist group &" + name + " not terminated"; return MRLBM_ENAMELIST; }
        groups[name] = clean.substr(ne, endg - ne);
        order.push_back(name);
        pos = endg + 1;
    }
    struct Var { const char* name; char type; void* ptr; };
    const std::map<std::string, std::vector<Var>> spec = {
        {"domainsize", {{"nx", 'i', &cfg.nx}, {"ny", 'i', &cfg.ny}, {"lattice_type", 'i', &cfg.lattice_type}}},
        {"cylinder", {{"ncy", 'i', &cfg.ncy}, {"l_front", 'i', &cfg.L_front}, {"l_back", 'i', &cfg.L_back},
                      {"l_top", 'i', &cfg.L_top}, {"l_bot", 'i', &cfg.L_bot}}},
        {"numbers", {{"re", 'r', &cfg.Re}}},
        {"parallel", {{"num_threads", 'i', &cfg.num_threads}}},
        {"controls", {{"uo", 'r', &cfg.uo}, {"rho_infty", 'r', &cfg.rho_infty}, {"iplot", 'i', &cfg.iplot},
                      {"max_iter", 'i', &cfg.max_iter}, {"isave", 'i', &cfg.isave}, {"irestart", 'i', &cfg.irestart},
                      {"statsbegin", 'i', &cfg.statsbegin}, {"statsend", 'i', &cfg.statsend},
                      {"iplotstats", 'i', &cfg.iplotstats}}},
        {"logicalcontrols", {{"post_process", 'l', &cfg.post_process}, {"x_periodic", 'l', &cfg.x_periodic},
                             {"y_periodic", 'l', &cfg.y_periodic},
                             {"channel_with_cylinder", 'l', &cfg.channel_with_cylinder},
                             {"channel_with_square", 'l', &cfg.channel_with_square}, {"incomp_bc", 'l', &cfg.incomp_bc},
                             {"incomp_bulk", 'l', &cfg.incomp_bulk}, {"vel_interp", 'l', &cfg.vel_interp},
                             {"mom_interp", 'l', &cfg.mom_interp}, {"rotated_coordinate", 'l', &cfg.rotated_coordinate},
                             {"strong_mass_bc", 'l', &cfg.strong_mass_bc}, {"eq_mass_bc", 'l', &cfg.eq_mass_bc},
                             {"weak_mass_bc", 'l', &cfg.weak_mass_bc}}},
    };
    // the reference reads the groups in this order and stops on the first failure
    const char* need[] = {"domainsize", "cylinder", "numbers", "parallel", "controls", "logicalcontrols"};
    for (const char* gname : need) {
        auto it = groups.find(gname);
        if (it == groups.end()) { err = std::string("namelist group &") + gname + " missing"; return MRLBM_ENAMELIST; }
        const auto& vars = spec.at(gname);
        std::string body = it->second;
        for (auto& ch : body) if (ch == '\n' || ch == '\r' || ch == '\t') ch = ' ';
        // items are name = value separated by commas or blanks
        size_t p = 0;
        while (true) {
            size_t eq = body.find('=', p);
            if (eq == std::string::npos) {
                if (!trim(body.substr(p)).empty() && trim(body.substr(p)) != ",") {
                    err = std::string("malformed item in &") + gname;
                    return MRLBM_ENAMELIST;
                }
                break;
            }
            std::string name = lower(trim(body.substr(p, eq - p)));
            while (!name.empty() && (name[0] == ',' || name[0] == ' ')) name = trim(name.substr(1));
            size_t next_eq = body.find('=', eq + 1);
            size_t vend = body.size();
            if (next_eq != std::string::npos) {
                // value ends at the separator before the next name
                size_t k = next_eq;
                while (k > eq && body[k - 1] == ' ') --k;
                while (k > eq && body[k - 1] != ' ' && body[k - 1] != ',') --k;
                vend = k;
            }
            std::string val = trim(body.substr(eq + 1, vend - eq - 1));
            while (!val.empty() && val.back() == ',') val = trim(val.substr(0, val.size() - 1));
            p = vend;
            const Var* v = nullptr;
            for (const auto& x : vars) if (name == x.name) v = &x;
            if (!v) { err = "unknown variable '" + name + "' in &" + gname; return MRLBM_ENAMELIST; }
            bool ok = false;
            if (v->type == 'i') ok = parse_int(val, *(int32_t*)v->ptr);
            else if (v->type == 'r') ok = parse_real(val, *(double*)v->ptr);
            else ok = parse_logical(val, *(int32_t*)v->ptr);
            if (!ok) { err = "bad value '" + val + "' for " + name + " in &" + gname; return MRLBM_ENAMELIST; }
            if (next_eq == std::string::npos) break;
        }
    }
    return MRLBM_OK;
}

// ---------------------------------------------------------------------------------------
namespace {
inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
inline double unit_open(uint64_t seed, uint64_t counter) {
    const uint64_t r = splitmix64(seed ^ splitmix64(counter));
    return ((double)(r >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
// standard normal for node n, component c (Box-Muller on two SplitMix64 draws)
inline double gauss(uint64_t seed, uint64_t n, int c) {
    const double u1 = unit_open(seed, 4 * n + 2 * (uint64_t)c);
    const double u2 = unit_open(seed, 4 * n + 2 * (uint64_t)c + 1);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}
}  // namespace

void initial_state(const mrlbm_config& cfg, const Lattice64& lat, int nx, int ny, std::vector<double>& f) {
    const size_t N = (size_t)nx * ny;
    f.assign(N * Q, 0.0);
    const double U = cfg.uo;
    for (size_t n = 0; n < N; ++n) {
        if (cfg.init_mode == MRLBM_INIT_NOISE) {
            // rho = 1, u = (U,0) + noise; populations from the regularized form with m = u u
            const double u = U + cfg.noise_amp * U * gauss(cfg.seed, n, 0);
            const double v = cfg.noise_amp * U * gauss(cfg.seed, n, 1);
            const double mxx = u * u, myy = v * v, mxy = u * v;
            for (int k = 0; k < Q; ++k) {
                const double cu = (double)ex(k) * u + (double)ey(k) * v;
                f[n + N * k] = lat.w[k] * 1.0 * (1.0 + (3.0 * cu) + 4.50 * mxx * lat.hxx[k] +
                                                 4.50 * myy * lat.hyy[k] + 9.00 * mxy * lat.hxy[k]);
            }
        } else {
            for (int k = 0; k < Q; ++k) f[n + N * k] = lat.w[k] * 1.0;        // 2d_mrlbm.f90:1231
        }
    }
}

}  // namespace mrlbm
