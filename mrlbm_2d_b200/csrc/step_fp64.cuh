// step_fp64.cuh -- FP64 fused time step, arithmetic in the reference's exact order.
//
// One launch advances one time step of 2d_mrlbm.f90:231-535.  State between launches is
// the post-collision population field fout (plus a ghost ring for populations the
// reference never overwrites).  A launch has two kinds of blocks:
//   * boundary blocks (the first nbblk): one thread per curved-wall boundary node.  Each
//     pulls its own populations and those of its 8 bilinear-stencil nodes from the previous
//     fout, recomputes the stencil moments, extrapolates velocity and rotated moments,
//     runs the regularized closure, collides, stores, and computes the momentum-exchange
//     force; forces and the inlet density sum are reduced with warp shuffles and the last
//     boundary block to arrive writes one record per step.
//   * bulk tiles: one thread per node and row of the tile; pull-stream, moments, edge
//     Dirichlet values and regularized edge closures, moment-space collision, Hermite
//     reconstruction, coalesced store.  Boundary nodes are skipped (the boundary blocks
//     own them); solid nodes are ordinary nodes, as in the reference.
// Every expression follows the reference's operation order (sums from k = 0 upwards,
// products left to right); the translation unit is compiled with -fmad=false, so each
// node's result is bit-identical to the reference's FP64 arithmetic.
#pragma once
#include <cuda_runtime.h>
#include "step_common.cuh"

namespace mrlbm {
namespace fp64 {

using P = StepParams<double>;

struct Mac { double rho, ux, uy, mxx, myy, mxy; };

// Macroscopic variables, 2d_mrlbm.f90:235-242.
__device__ __forceinline__ Mac moments(const double f[Q], double hm, double hp) {
    Mac m;
    double s = f[0];
    s = s + f[1]; s = s + f[2]; s = s + f[3]; s = s + f[4];
    s = s + f[5]; s = s + f[6]; s = s + f[7]; s = s + f[8];
    m.rho = s;
    const double inv_rho = 1.0 / s;
    const double sx = ((((f[1] - f[3]) + f[5]) - f[6]) - f[7]) + f[8];
    const double sy = ((((f[2] - f[4]) + f[5]) + f[6]) - f[7]) - f[8];
    double sxx = f[0] * hm;
    sxx = sxx + f[1] * hp; sxx = sxx + f[2] * hm; sxx = sxx + f[3] * hp; sxx = sxx + f[4] * hm;
    sxx = sxx + f[5] * hp; sxx = sxx + f[6] * hp; sxx = sxx + f[7] * hp; sxx = sxx + f[8] * hp;
    double syy = f[0] * hm;
    syy = syy + f[1] * hm; syy = syy + f[2] * hp; syy = syy + f[3] * hm; syy = syy + f[4] * hp;
    syy = syy + f[5] * hp; syy = syy + f[6] * hp; syy = syy + f[7] * hp; syy = syy + f[8] * hp;
    const double sxy = ((f[5] - f[6]) + f[7]) - f[8];
    m.ux = sx * inv_rho;
    m.uy = sy * inv_rho;
    m.mxx = sxx * inv_rho;
    m.myy = syy * inv_rho;
    m.mxy = sxy * inv_rho;
    return m;
}

// rho, ux, uy only (outlet copy source and stencil velocities).
__device__ __forceinline__ void moments_u(const double f[Q], double& rho, double& ux, double& uy) {
    double s = f[0];
    s = s + f[1]; s = s + f[2]; s = s + f[3]; s = s + f[4];
    s = s + f[5]; s = s + f[6]; s = s + f[7]; s = s + f[8];
    rho = s;
    const double inv_rho = 1.0 / s;
    ux = (((((f[1] - f[3]) + f[5]) - f[6]) - f[7]) + f[8]) * inv_rho;
    uy = (((((f[2] - f[4]) + f[5]) + f[6]) - f[7]) - f[8]) * inv_rho;
}

// Hxx_k and Hyy_k as values hm / hp.
__device__ __forceinline__ double hxx_of(int k, double hm, double hp) { return ex(k) != 0 ? hp : hm; }
__device__ __forceinline__ double hyy_of(int k, double hm, double hp) { return ey(k) != 0 ? hp : hm; }

// Sums over a fixed incoming mask, normalised by rho_I (prologue of apply_bc,
// 2d_mrlbm.f90:1249-1269).
template <int MASK>
__device__ __forceinline__ void incoming(const double f[Q], double hm, double hp, double& rhoI, double& mxxI,
                                         double& myyI, double& mxyI) {
    bool first = true;
    double r = 0.0, a = 0.0, b = 0.0, c = 0.0;
    bool cfirst = true;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        if (!((MASK >> k) & 1)) continue;
        if (first) {
            r = f[k];
            a = f[k] * hxx_of(k, hm, hp);
            b = f[k] * hyy_of(k, hm, hp);
            first = false;
        } else {
            r = r + f[k];
            a = a + f[k] * hxx_of(k, hm, hp);
            b = b + f[k] * hyy_of(k, hm, hp);
        }
        const int hxy = ex(k) * ey(k);
        if (hxy != 0) {
            if (cfirst) { c = hxy > 0 ? f[k] : -f[k]; cfirst = false; }
            else c = hxy > 0 ? c + f[k] : c - f[k];
        }
    }
    rhoI = r;
    const double inv = 1.0 / rhoI;
    mxxI = a * inv;
    myyI = b * inv;
    mxyI = c * inv;
}

// Masks (bit k = population k) of apply_bc's Is vectors (2d_mrlbm.f90:1254, 1283, 1311, 1339).
constexpr int M_OUTLET = (1 << 0) | (1 << 1) | (1 << 2) | (1 << 4) | (1 << 5) | (1 << 8);
constexpr int M_INLET = (1 << 0) | (1 << 2) | (1 << 3) | (1 << 4) | (1 << 6) | (1 << 7);
constexpr int M_TOP = (1 << 0) | (1 << 1) | (1 << 2) | (1 << 3) | (1 << 5) | (1 << 6);
constexpr int M_BOTTOM = (1 << 0) | (1 << 1) | (1 << 3) | (1 << 4) | (1 << 7) | (1 << 8);

// Edge nodes: Dirichlet values (2d_mrlbm.f90:249-272) then the regularized closure the
// reference applies last at this node (apply_bc / apply_bc_incomp, 2d_mrlbm.f90:313-351).
__device__ __forceinline__ void edge_node(const P& p, int i, int j, const double f[Q], Mac& m) {
    const int nx = p.L.nx, ny = p.L.ny;
    const bool outlet = !p.xper && !p.halo_r && i == nx;
    const bool inlet = !p.xper && !p.halo_l && i == 1;
    const bool top = p.walls_ref && j == ny;
    const bool bottom = p.walls_ref && j == 1;
    if (outlet) {
        double fn[Q];
        gather(p, nx - 1, j, fn);
        moments_u(fn, m.rho, m.ux, m.uy);
    }
    if (inlet) {
        m.ux = p.u_in ? p.u_in[j - 1] : p.uinlet;
        m.uy = p.vinlet;
    }
    if (top || bottom) { m.ux = 0.0; m.uy = 0.0; }
    const double hm = p.hm, hp = p.hp, omega = p.omega;
    double rhoI, mxxI, myyI, mxyI;
    if (top || bottom) {
        if (top) incoming<M_TOP>(f, hm, hp, rhoI, mxxI, myyI, mxyI);
        else incoming<M_BOTTOM>(f, hm, hp, rhoI, mxxI, myyI, mxyI);
        if (!p.incomp_bc) {
            m.rho = 3.0 * rhoI * (4.0 + 3.0 * (1.0 - omega) * myyI) / (9.0 + omega);
            const double rp = m.rho;
            m.mxx = 6.0 * rhoI * mxxI / (5.0 * rp);
            m.myy = (rp + 9.0 * rhoI * myyI) / (6.0 * rp);
            m.mxy = 2.0 * rhoI * mxyI / rp;
        } else {
            m.rho = 6.0 * rhoI / 5.0;
            m.mxx = 0.0;
            m.myy = 0.0;
            m.mxy = 5.0 * mxyI / 3.0;
        }
    } else if (inlet) {
        incoming<M_INLET>(f, hm, hp, rhoI, mxxI, myyI, mxyI);
        if (!p.incomp_bc) {
            m.rho = (4.0 * rhoI + 3.0 * rhoI * mxxI) / (3.0 - 3.0 * m.ux);
            const double rp = m.rho;
            m.mxx = (rp + 9.0 * rhoI * mxxI + 3.0 * rp * m.ux) / (6.0 * rp);
            m.myy = 6.0 * rhoI * myyI / (5.0 * rp);
            m.mxy = 2.0 * rhoI * mxyI / rp;
        } else {
            m.rho = 6.0 * rhoI / (5.0 - 3.0 * m.ux - 3.0 * (m.ux * m.ux));
            const double rp = m.rho;
            m.mxx = m.ux * m.ux;
            m.myy = 0.0;
            m.mxy = 2.0 * rhoI * mxyI / rp;
        }
    } else if (outlet) {
        incoming<M_OUTLET>(f, hm, hp, rhoI, mxxI, myyI, mxyI);
        const double rp = m.rho;
        if (!p.incomp_bc) {
            m.mxx = (rp + 9.0 * rhoI * mxxI - 3.0 * rp * m.ux) / (6.0 * rp);
            m.myy = 6.0 * rhoI * myyI / (5.0 * rp);
            m.mxy = (6.0 * rhoI * mxyI - rp * m.uy) / (3.0 * rp);
        } else {
            m.mxx = m.ux * m.ux;
            m.myy = m.uy * m.uy;
            m.mxy = (6.0 * rhoI * mxyI - rp * m.uy) / (3.0 * rp);
        }
    }
}

// Moment-space collision (2d_mrlbm.f90:407-415, 419-428) and Hermite reconstruction
// (2d_mrlbm.f90:445-457), per direction in the reference's left-to-right order.
__device__ __forceinline__ void collide(const P& p, const Mac& m, double fo[Q]) {
    const double om = p.omega, om1 = p.omega1;
    double mxx = om1 * m.mxx + om * m.ux * m.ux;
    double myy = om1 * m.myy + om * m.uy * m.uy;
    double mxy = om1 * m.mxy + om * m.ux * m.uy;
    if (p.incomp_bulk) {
        const double t = 0.50 * (mxx + myy - m.ux * m.ux - m.uy * m.uy);
        mxx = mxx - t;
        myy = myy - t;
    }
    const double a = 4.50 * mxx, b = 4.50 * myy, c = 9.00 * mxy;
    const double am = a * p.hm, ap = a * p.hp, bm = b * p.hm, bp = b * p.hp;
    const double t1 = 3.0 * m.ux, t2 = 3.0 * m.uy;
    const double t5 = 3.0 * (m.ux + m.uy), t8 = 3.0 * (m.ux - m.uy);
    const double w0 = p.w[0] * m.rho, w1 = p.w[1] * m.rho, w5 = p.w[5] * m.rho;
    fo[0] = w0 * ((1.0 + am) + bm);
    fo[1] = w1 * (((1.0 + t1) + ap) + bm);
    fo[2] = w1 * (((1.0 + t2) + am) + bp);
    fo[3] = w1 * (((1.0 - t1) + ap) + bm);
    fo[4] = w1 * (((1.0 - t2) + am) + bp);
    fo[5] = w5 * ((((1.0 + t5) + ap) + bp) + c);
    fo[6] = w5 * ((((1.0 - t8) + ap) + bp) - c);
    fo[7] = w5 * ((((1.0 - t5) + ap) + bp) + c);
    fo[8] = w5 * ((((1.0 + t8) + ap) + bp) - c);
}

// Post-boundary-condition macroscopic values of a non-cylinder node.
__device__ __forceinline__ Mac node_macro(const P& p, int i, int j, const double f[Q]) {
    Mac m = moments(f, p.hm, p.hp);
    if (!is_interior(p, i, j)) edge_node(p, i, j, f, m);
    return m;
}

// ---------------------------------------------------------------------------------------
// Curved-wall boundary node (2d_mrlbm.f90:294-311 and the routines they call).

// Velocity and rotated second moments (2d_mrlbm.f90:842-867) of one bilinear stencil node.
__device__ __forceinline__ void stencil_node(const P& p, int si, int sj, double cc, double ss, double s2, double& ux,
                                             double& uy, double& mx, double& my) {
    double f[Q];
    gather(p, si, sj, f);
    const Mac m = moments(f, p.hm, p.hp);
    ux = m.ux;
    uy = m.uy;
    mx = m.mxx * cc + m.myy * ss + m.mxy * s2;
    my = m.mxx * ss + m.myy * cc - m.mxy * s2;
}

// Rotated closures, 2d_mrlbm.f90:1635-1765 (strong), 1873-1972 (rhoeq), 1767-1871 (weak).
__device__ __forceinline__ void closure_rotated_body(const P& p, const BTab<double>& tb, int li, const double f[Q], double uxp,
                                                     double uyp, double Mxx, double Myy, Mac& m) {
    const int Is = tb.gi(I_IS, li), Os = tb.gi(I_OS, li);
    const double omega = p.omega;
    const int variant = p.closure;
    double rhoI = 0, mxxI = 0, myyI = 0, mxyI = 0, A_p = 0, E_p = 0;
    double B11 = 0, B22 = 0, B12 = 0, D_xy = 0, F11_xy = 0, F22_xy = 0, F12_xy = 0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double cxp = tb.gf(G_CXP + k, li), cyp = tb.gf(G_CYP + k, li);
        const double hxx = tb.gf(G_HXXP + k, li), hyy = tb.gf(G_HYYP + k, li), hxy = tb.gf(G_HXYP + k, li);
        const double wk = p.w[k];
        const double A_i = wk * (1.0 + 3.0 * uxp * cxp + 3.0 * uyp * cyp);
        const double E_i = wk * (1.0 + 3.0 * uxp * cxp + 3.0 * uyp * cyp + 4.50 * (uxp * uxp) * hxx +
                                 4.50 * (uyp * uyp) * hyy + 9.0 * (uxp * uyp) * hxy);
        const double B11_i = 4.50 * wk * hxx, B22_i = 4.50 * wk * hyy, B12_i = 4.50 * wk * hxy;
        const bool o = (Os >> k) & 1, in = (Is >> k) & 1;
        if (variant == CLOSURE_STRONG) {
            if (o) { A_p = A_p + A_i; E_p = E_p + E_i; B11 = B11 + B11_i; B22 = B22 + B22_i; B12 = B12 + B12_i; }
        }
        if (in) {
            rhoI = rhoI + f[k];
            mxxI = mxxI + f[k] * hxx;
            myyI = myyI + f[k] * hyy;
            mxyI = mxyI + f[k] * hxy;
            if (variant == CLOSURE_WEAK) { A_p = A_p + A_i; B11 = B11 + B11_i; B22 = B22 + B22_i; B12 = B12 + B12_i; }
            if (variant == CLOSURE_RHOEQ) E_p = E_p + E_i;
            D_xy = D_xy + A_i * hxy;
            F11_xy = F11_xy + B11_i * hxy;
            F22_xy = F22_xy + B22_i * hxy;
            F12_xy = F12_xy + B12_i * hxy;
        }
    }
    const double inv = 1.0 / rhoI;
    mxxI = mxxI * inv;
    myyI = myyI * inv;
    mxyI = mxyI * inv;
    double Mxy, rhop;
    if (variant == CLOSURE_STRONG) {
        const double G_p = (1.0 - omega) * A_p + omega * E_p;
        const double J11 = (1.0 - omega) * B11, J22 = (1.0 - omega) * B22, J12 = (1.0 - omega) * B12;
        const double L11 = J11 * mxyI - F11_xy, L22 = J22 * mxyI - F22_xy, L12 = 2.0 * (J12 * mxyI - F12_xy);
        const double R = D_xy - G_p * mxyI;
        Mxy = (R - Mxx * L11 - Myy * L22) / L12;
        const double den = (1.0 - omega) * A_p + (1.0 - omega) * (Mxx * B11 + Myy * B22 + 2.0 * Mxy * B12) + omega * E_p;
        rhop = rhoI / den;
    } else if (variant == CLOSURE_WEAK) {
        const double L11 = B11 * mxyI - F11_xy, L22 = B22 * mxyI - F22_xy, L12 = 2.0 * (B12 * mxyI - F12_xy);
        const double R = D_xy - A_p * mxyI;
        Mxy = (R - Mxx * L11 - Myy * L22) / L12;
        const double den = A_p + (Mxx * B11 + Myy * B22 + 2.0 * Mxy * B12);
        rhop = rhoI / den;
    } else {  // CLOSURE_RHOEQ
        const double L11 = F11_xy, L22 = F22_xy, L12 = 2.0 * F12_xy;
        const double R = E_p * mxyI - D_xy;
        Mxy = (R - Mxx * L11 - Myy * L22) / L12;
        rhop = rhoI / E_p;
    }
    const double cc = tb.gf(G_CC, li), ss = tb.gf(G_SS, li), s2 = tb.gf(G_S2TH, li), c2 = tb.gf(G_C2TH, li);
    m.rho = rhop;
    m.mxx = Mxx * cc + Myy * ss - Mxy * s2;
    m.myy = Mxx * ss + Myy * cc + Mxy * s2;
    m.mxy = (Mxx - Myy) * 0.50 * s2 + Mxy * c2;
}

static __device__ __noinline__ void closure_rotated(const P& p, const BTab<double>& tb, int li, const double f[Q], double uxp, double uyp,
                                                    double Mxx, double Myy, Mac& m) {
    closure_rotated_body(p, tb, li, f, uxp, uyp, Mxx, Myy, m);
}

// Unrotated closure with Cramer's rule, 2d_mrlbm.f90:1496-1633 and 1974-2003.
static __device__ __noinline__ void closure_unrotated(const P& p, const BTab<double>& tb, int li, const double f[Q], double uxp,
                                                      double uyp, Mac& m) {
    const int Is = tb.gi(I_IS, li), Os = tb.gi(I_OS, li);
    const double omega = p.omega, hm = p.hm, hp = p.hp;
    double rhoI = 0, mxxI = 0, myyI = 0, mxyI = 0, A_p = 0, E_p = 0, B11 = 0, B22 = 0, B12 = 0;
    double D_xx = 0, D_yy = 0, D_xy = 0, F11_xx = 0, F12_xx = 0, F22_xx = 0, F11_yy = 0, F12_yy = 0, F22_yy = 0;
    double F11_xy = 0, F12_xy = 0, F22_xy = 0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double hxx = hxx_of(k, hm, hp), hyy = hyy_of(k, hm, hp), hxy = (double)(ex(k) * ey(k));
        const double wk = p.w[k];
        const double A_i = wk * (1.0 + 3.0 * uxp * (double)ex(k) + 3.0 * uyp * (double)ey(k));
        const double E_i = wk * (1.0 + 3.0 * uxp * (double)ex(k) + 3.0 * uyp * (double)ey(k) + 4.50 * (uxp * uxp) * hxx +
                                 4.50 * (uyp * uyp) * hyy + 9.0 * (uxp * uyp) * hxy);
        const double B11_i = 4.50 * wk * hxx, B22_i = 4.50 * wk * hyy, B12_i = 4.50 * wk * hxy;
        if ((Os >> k) & 1) { A_p = A_p + A_i; E_p = E_p + E_i; B11 = B11 + B11_i; B22 = B22 + B22_i; B12 = B12 + B12_i; }
        if ((Is >> k) & 1) {
            rhoI = rhoI + f[k];
            mxxI = mxxI + f[k] * hxx;
            myyI = myyI + f[k] * hyy;
            mxyI = mxyI + f[k] * hxy;
            D_xx = D_xx + A_i * hxx; D_yy = D_yy + A_i * hyy; D_xy = D_xy + A_i * hxy;
            F11_xx = F11_xx + B11_i * hxx; F22_xx = F22_xx + B22_i * hxx; F12_xx = F12_xx + B12_i * hxx;
            F11_yy = F11_yy + B11_i * hyy; F22_yy = F22_yy + B22_i * hyy; F12_yy = F12_yy + B12_i * hyy;
            F11_xy = F11_xy + B11_i * hxy; F22_xy = F22_xy + B22_i * hxy; F12_xy = F12_xy + B12_i * hxy;
        }
    }
    const double inv = 1.0 / rhoI;
    mxxI = mxxI * inv;
    myyI = myyI * inv;
    mxyI = mxyI * inv;
    const double G_p = (1.0 - omega) * A_p + omega * E_p;
    const double J11 = (1.0 - omega) * B11, J22 = (1.0 - omega) * B22, J12 = (1.0 - omega) * B12;
    const double a1 = J11 * mxxI - F11_xx, b1 = J22 * mxxI - F22_xx, c1 = 2.0 * (J12 * mxxI - F12_xx);
    const double a2 = J11 * myyI - F11_yy, b2 = J22 * myyI - F22_yy, c2 = 2.0 * (J12 * myyI - F12_yy);
    const double a3 = J11 * mxyI - F11_xy, b3 = J22 * mxyI - F22_xy, c3 = 2.0 * (J12 * mxyI - F12_xy);
    const double d1 = D_xx - G_p * mxxI, d2 = D_yy - G_p * myyI, d3 = D_xy - G_p * mxyI;
    const double denom = a3 * b2 * c1 - a2 * b3 * c1 - a3 * b1 * c2 + a1 * b3 * c2 + a2 * b1 * c3 - a1 * b2 * c3;
    const double Mxx = -((-b3 * c2 * d1 + b2 * c3 * d1 + b3 * c1 * d2 - b1 * c3 * d2 - b2 * c1 * d3 + b1 * c2 * d3) / denom);
    const double Myy = -((a3 * c2 * d1 - a2 * c3 * d1 - a3 * c1 * d2 + a1 * c3 * d2 + a2 * c1 * d3 - a1 * c2 * d3) / denom);
    const double Mxy = -((-a3 * b2 * d1 + a2 * b3 * d1 + a3 * b1 * d2 - a1 * b3 * d2 - a2 * b1 * d3 + a1 * b2 * d3) / denom);
    const double den = (1.0 - omega) * A_p + (1.0 - omega) * (Mxx * B11 + Myy * B22 + 2.0 * Mxy * B12) + omega * E_p;
    m.rho = rhoI / den;
    m.mxx = Mxx;
    m.myy = Myy;
    m.mxy = Mxy;
}

// Lane 0 of a boundary node: extrapolated velocity / rotated moments from the reference
// points (the wall value is 0; 2d_mrlbm.f90:809-814, 919-924), closure, collision, store,
// momentum-exchange force (evaluate_forces, 2d_mrlbm.f90:558-591).  PRE: the node's
// populations were gathered by the caller (fpre) and every call below is inlined, so nothing
// of the node goes through local memory; without PRE (kernels with few registers per thread)
// the node gathers its own populations and the closures stay out of line.
template <bool FULL, bool PRE>
__device__ __forceinline__ void boundary_close_core(const P& p, const BTab<double>& tb, int li, int l, const double* fpre,
                                                    double ux2, double uy2, double mx2, double my2, double ux3, double uy3,
                                                    double mx3, double my3, double& Fx, double& Fy) {
    const int i = tb.gi(I_NODEI, li), j = tb.gi(I_NODEJ, li);
    double f[Q];
    if (PRE) {
#pragma unroll
        for (int k = 0; k < Q; ++k) f[k] = fpre[k];
    } else {
        gather(p, i, j, f);
    }
    Mac m = moments(f, p.hm, p.hp);
    const bool rotated = p.closure != CLOSURE_UNROTATED;
    double mxxp = 0.0, myyp = 0.0;
    const double t1 = tb.gf(G_T1, li), t2 = tb.gf(G_T2, li), t3 = tb.gf(G_T3, li);
    if (!rotated || p.vel_interp) {
        m.ux = t1 * 0.0 + t2 * ux2 - t3 * ux3;
        m.uy = t1 * 0.0 + t2 * uy2 - t3 * uy3;
    }
    if (rotated && p.mom_interp) {
        mxxp = t1 * 0.0 + t2 * mx2 - t3 * mx3;
        myyp = t1 * 0.0 + t2 * my2 - t3 * my3;
    }
    if (rotated) {
        if (p.closure != CLOSURE_NONE) {
            const double c = tb.gf(G_CTH, li), s = tb.gf(G_STH, li);
            const double uxp = m.ux * c + m.uy * s;    // 2d_mrlbm.f90:304-305
            const double uyp = m.uy * c - m.ux * s;
            if (PRE) closure_rotated_body(p, tb, li, f, uxp, uyp, mxxp, myyp, m);
            else closure_rotated(p, tb, li, f, uxp, uyp, mxxp, myyp, m);
        }
    } else {
        closure_unrotated(p, tb, li, f, m.ux, m.uy, m);
    }
    if (!(m.rho > 0.0)) flag_bad_density(p);
    if (FULL && p.macro) store_macro(p, i, j, m.rho, m.ux, m.uy, m.mxx, m.myy, m.mxy);
    if (FULL && p.fstat) accumulate_fields(p, i, j, m.rho, m.ux, m.uy);
    double fo[Q];
    collide(p, m, fo);
    store(p, i, j, fo);
    const int Is = tb.gi(I_IS, li), Os = tb.gi(I_OS, li);
    double fxo = 0.0, fyo = 0.0, fxi = 0.0, fyi = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        if ((Os >> k) & 1) { fxo = fxo + fo[k] * (double)ex(k); fyo = fyo + fo[k] * (double)ey(k); }
        if ((Is >> k) & 1) { fxi = fxi + f[k] * (double)ex(k); fyi = fyi + f[k] * (double)ey(k); }
    }
    Fx = fxi - fxo;
    Fy = fyi - fyo;
    if (p.node_force) { p.node_force[2 * l] = Fx; p.node_force[2 * l + 1] = Fy; }
}

template <bool FULL>
__device__ __noinline__ void boundary_close(const P& p, const BTab<double>& tb, int li, int l, double ux2, double uy2,
                                            double mx2, double my2, double ux3, double uy3, double mx3, double my3,
                                            double& Fx, double& Fy) {
    boundary_close_core<FULL, false>(p, tb, li, l, nullptr, ux2, uy2, mx2, my2, ux3, uy3, mx3, my3, Fx, Fy);
}

// Edge nodes (first/last row or column): own gather, Dirichlet values and closures.  Inline,
// so the populations stay in registers and the gathers of a node overlap (edge blocks are a
// branch of their own, so the bulk path's registers are not affected).
template <bool FULL>
__device__ __forceinline__ double edge_bulk_node(const P& p, int i, int j, int cls) {
    double f[Q];
    gather(p, i, j, f);
    Mac m = moments(f, p.hm, p.hp);
    edge_node(p, i, j, f, m);
    if ((cls == CLS_SOLID && p.zero_solid_u) || cls == CLS_SOLID_ZERO) { m.ux = 0.0; m.uy = 0.0; }
    if (!(m.rho > 0.0)) flag_bad_density(p);
    if (FULL && p.macro) store_macro(p, i, j, m.rho, m.ux, m.uy, m.mxx, m.myy, m.mxy);
    if (FULL && p.fstat) accumulate_fields(p, i, j, m.rho, m.ux, m.uy);
    double fo[Q];
    collide(p, m, fo);
    if (FULL && p.body) add_body_force(p, i, j, fo);
    store(p, i, j, fo);
    return m.rho;
}

// Bulk node (fluid or solid).
// Interior fluid or solid node: populations already gathered.
template <bool FULL>
__device__ __forceinline__ void compute(const P& p, int i, int j, int cls, const double f[Q], double fo[Q]) {
    FieldPre pre;
    if (FULL && p.fstat) fields_load(p, i, j, pre);
    Mac m = moments(f, p.hm, p.hp);
    if ((cls == CLS_SOLID && p.zero_solid_u) || cls == CLS_SOLID_ZERO) { m.ux = 0.0; m.uy = 0.0; }
    if (!(m.rho > 0.0)) flag_bad_density(p);
    if (FULL && p.macro) store_macro(p, i, j, m.rho, m.ux, m.uy, m.mxx, m.myy, m.mxy);
    if (FULL && p.fstat) fields_store(p, i, j, pre, m.rho, m.ux, m.uy);
    collide(p, m, fo);
    if (FULL && p.body) add_body_force(p, i, j, fo);
}

template <bool FULL>
__device__ __forceinline__ void finish(const P& p, int i, int j, int cls, const double f[Q]) {
    double fo[Q];
    compute<FULL>(p, i, j, cls, f, fo);
    store(p, i, j, fo);
}

// FULL: the node paths include the optional per-node work (field statistics, macroscopic
// output, body force), each behind its run-time switch.  The lean instantiation leaves it
// out; the launchers pick it when all three are off, which keeps the registers and the
// branches of that work out of the common step.
template <bool FULL>
struct PhysicsT {
    using P = StepParams<double>;
    using T = double;
    static __device__ __forceinline__ void compute(const P& p, int i, int j, int cls, const T f[Q], T fo[Q]) {
        fp64::compute<FULL>(p, i, j, cls, f, fo);
    }
    static __device__ __forceinline__ void finish(const P& p, int i, int j, int cls, const T f[Q]) {
        fp64::finish<FULL>(p, i, j, cls, f);
    }
    static __device__ __forceinline__ double edge_bulk_node(const P& p, int i, int j, int cls) {
        return fp64::edge_bulk_node<FULL>(p, i, j, cls);
    }
    static __device__ __forceinline__ void stencil_node(const P& p, int si, int sj, T cc, T ss, T s2, T& ux, T& uy,
                                                        T& mx, T& my) {
        fp64::stencil_node(p, si, sj, cc, ss, s2, ux, uy, mx, my);
    }
    static __device__ __forceinline__ void boundary_close(const P& p, const BTab<T>& tb, int li, int l, T ux2, T uy2,
                                                          T mx2, T my2, T ux3, T uy3, T mx3, T my3, double& Fx,
                                                          double& Fy) {
        fp64::boundary_close<FULL>(p, tb, li, l, ux2, uy2, mx2, my2, ux3, uy3, mx3, my3, Fx, Fy);
    }
    static __device__ __forceinline__ void boundary_close_pre(const P& p, const BTab<T>& tb, int li, int l, const T f[Q],
                                                              T ux2, T uy2, T mx2, T my2, T ux3, T uy3, T mx3, T my3,
                                                              double& Fx, double& Fy) {
        fp64::boundary_close_core<FULL, true>(p, tb, li, l, f, ux2, uy2, mx2, my2, ux3, uy3, mx3, my3, Fx, Fy);
    }
    // registers per thread a kernel needs before its wall-node path is inlined (boundary_close_pre)
    static constexpr int WIDE_REGS = 128;
    static constexpr bool FUSED_AUX = false;         // the wall closures get a launch of their own
};
using Physics = PhysicsT<true>;
using PhysicsLean = PhysicsT<false>;

}  // namespace fp64
}  // namespace mrlbm
