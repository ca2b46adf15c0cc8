// step_fp32.cuh -- FP32 fused step in deviation form.
//
// Storage: g_k = f_k - w_k in FP32, w_k the reference's single-rounded weights
// (2d_mrlbm.f90:129), which are exact FP32 values.  Arithmetic is FP32 on small quantities
// only: every closure of the FP64 step (2d_mrlbm.f90:232-457) is rearranged so the
// rest-state parts that cancel (sums of w_k over fixed link sets, which are exact in real
// arithmetic but not with single-rounded weights) are folded into constants computed once
// in FP64 on the host (DevConsts).  The mass drift the reference has because
// sum(w) = 1 + 7.45e-9 is kept (eps_mass).  Forces are accumulated in FP64 from
// w_k + g_k.  Every curved-wall closure of the FP64 step has an FP32 form (rotated strong,
// weak and rho_eq, unrotated with Cramer's rule, none).
#pragma once
#include "step_common.cuh"

namespace mrlbm {
namespace fp32 {

using P = StepParams<float>;

struct Mac { float drho, rho, ux, uy, mxx, myy, mxy; };

constexpr float THIRD = 1.0f / 3.0f;

// 1 / x by the hardware approximation (PTX rcp.approx.ftz.f32, within one unit in the last
// place): the FP32 form is held to accuracy bounds against the FP64 step, not to a rounding
// pattern, and a node's density is near 1.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// rho = 1 + sum g + (sum w - 1); u = sum f c / rho; m = sum f H / rho with
// sum f H_xx = (sum_k w_k H_xx,k) + sum g c_x^2 - sum g / 3.
__device__ __forceinline__ Mac moments(const P& p, const float g[Q]) {
    Mac m;
    const float dg = (((g[0] + g[1]) + (g[2] + g[3])) + ((g[4] + g[5]) + (g[6] + g[7]))) + g[8];
    m.drho = dg + p.dc.eps_mass;
    m.rho = 1.0f + m.drho;
    const float inv = rcp_approx(m.rho);
    const float jx = ((g[1] - g[3]) + (g[5] - g[7])) + (g[8] - g[6]);
    const float jy = ((g[2] - g[4]) + (g[5] - g[7])) + (g[6] - g[8]);
    const float d4 = (g[5] + g[6]) + (g[7] + g[8]);
    const float sxx = (g[1] + g[3]) + d4;
    const float syy = (g[2] + g[4]) + d4;
    const float sxy = (g[5] - g[6]) + (g[7] - g[8]);
    m.ux = jx * inv;
    m.uy = jy * inv;
    m.mxx = ((sxx - THIRD * dg) + p.dc.cxx) * inv;
    m.myy = ((syy - THIRD * dg) + p.dc.cyy) * inv;
    m.mxy = sxy * inv;
    return m;
}

__device__ __forceinline__ float hxx_of(int k, float hm, float hp) { return ex(k) != 0 ? hp : hm; }
__device__ __forceinline__ float hyy_of(int k, float hm, float hp) { return ey(k) != 0 ? hp : hm; }

// Deviation sums over a fixed incoming mask: G = sum g, S_ab = sum g H_ab.
template <int MASK>
__device__ __forceinline__ void incoming(const float g[Q], float hm, float hp, float& G, float& Sxx, float& Syy,
                                         float& Sxy) {
    G = 0.f; Sxx = 0.f; Syy = 0.f; Sxy = 0.f;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        if (!((MASK >> k) & 1)) continue;
        G += g[k];
        Sxx += g[k] * hxx_of(k, hm, hp);
        Syy += g[k] * hyy_of(k, hm, hp);
        const int hxy = ex(k) * ey(k);
        if (hxy > 0) Sxy += g[k];
        if (hxy < 0) Sxy -= g[k];
    }
}

constexpr int M_OUTLET = (1 << 0) | (1 << 1) | (1 << 2) | (1 << 4) | (1 << 5) | (1 << 8);
constexpr int M_INLET = (1 << 0) | (1 << 2) | (1 << 3) | (1 << 4) | (1 << 6) | (1 << 7);
constexpr int M_TOP = (1 << 0) | (1 << 1) | (1 << 2) | (1 << 3) | (1 << 5) | (1 << 6);
constexpr int M_BOTTOM = (1 << 0) | (1 << 1) | (1 << 3) | (1 << 4) | (1 << 7) | (1 << 8);

// Edge nodes: Dirichlet values and the regularized edge closures of apply_bc /
// apply_bc_incomp (2d_mrlbm.f90:249-272, 1237-1494) in deviation form.
__device__ __forceinline__ void edge_node(const P& p, int i, int j, const float g[Q], Mac& m) {
    const int nx = p.L.nx, ny = p.L.ny;
    const bool outlet = !p.xper && !p.halo_r && i == nx;
    const bool inlet = !p.xper && !p.halo_l && i == 1;
    const bool top = p.walls_ref && j == ny;
    const bool bottom = p.walls_ref && j == 1;
    const DevConsts& c = p.dc;
    if (outlet) {                                   // rho, u copied from column nx-1
        float gn[Q];
        gather(p, nx - 1, j, gn);
        const Mac mn = moments(p, gn);
        m.drho = mn.drho; m.rho = mn.rho; m.ux = mn.ux; m.uy = mn.uy;
    }
    if (inlet) {
        m.ux = p.u_in ? p.u_in[j - 1] : p.uinlet;
        m.uy = p.vinlet;
    }
    if (top || bottom) { m.ux = 0.f; m.uy = 0.f; }
    const float hm = p.hm, hp = p.hp, om = p.omega;
    float G, Sxx, Syy, Sxy;
    if (top || bottom) {
        const int e = top ? 0 : 1;
        if (top) incoming<M_TOP>(g, hm, hp, G, Sxx, Syy, Sxy);
        else incoming<M_BOTTOM>(g, hm, hp, G, Sxx, Syy, Sxy);
        if (!p.incomp_bc) {
            m.drho = (c.k_w_rho[e] + 12.0f * G + 9.0f * (1.0f - om) * Syy) / (9.0f + om);
            m.rho = 1.0f + m.drho;
            m.mxx = 6.0f * (c.sw_w_xx[e] + Sxx) / (5.0f * m.rho);
            m.myy = (c.k_w_myy[e] + m.drho + 9.0f * Syy) / (6.0f * m.rho);
            m.mxy = 2.0f * Sxy / m.rho;
        } else {
            m.drho = (c.k_w_rho_inc[e] + 6.0f * G) / 5.0f;
            m.rho = 1.0f + m.drho;
            m.mxx = 0.f;
            m.myy = 0.f;
            m.mxy = 5.0f * (Sxy / (c.w_wall[e] + G)) / 3.0f;
        }
    } else if (inlet) {
        incoming<M_INLET>(g, hm, hp, G, Sxx, Syy, Sxy);
        const float u = m.ux;
        if (!p.incomp_bc) {
            m.drho = (c.k_in_rho + 4.0f * G + 3.0f * Sxx + 3.0f * u) / (3.0f - 3.0f * u);
            m.rho = 1.0f + m.drho;
            m.mxx = (c.k_in_mxx + m.drho + 9.0f * Sxx + 3.0f * m.rho * u) / (6.0f * m.rho);
            m.myy = 6.0f * (c.sw_in_yy + Syy) / (5.0f * m.rho);
            m.mxy = 2.0f * Sxy / m.rho;
        } else {
            m.drho = (c.k_in_rho_inc + 6.0f * G + 3.0f * u + 3.0f * (u * u)) / (5.0f - 3.0f * u - 3.0f * (u * u));
            m.rho = 1.0f + m.drho;
            m.mxx = u * u;
            m.myy = 0.f;
            m.mxy = 2.0f * Sxy / m.rho;
        }
    } else if (outlet) {
        incoming<M_OUTLET>(g, hm, hp, G, Sxx, Syy, Sxy);
        const float rp = m.rho;
        if (!p.incomp_bc) {
            m.mxx = (c.k_out_mxx + m.drho + 9.0f * Sxx - 3.0f * rp * m.ux) / (6.0f * rp);
            m.myy = 6.0f * (c.sw_out_yy + Syy) / (5.0f * rp);
        } else {
            m.mxx = m.ux * m.ux;
            m.myy = m.uy * m.uy;
        }
        m.mxy = (6.0f * Sxy - rp * m.uy) / (3.0f * rp);
    }
}

// Moment-space collision and Hermite reconstruction (2d_mrlbm.f90:407-457) on deviations:
// g_out_k = w_k (drho + rho a_k), a_k = 3 c_k.u + 4.5 m_xx H_xx,k + 4.5 m_yy H_yy,k + 9 m_xy H_xy,k.
__device__ __forceinline__ void collide(const P& p, const Mac& m, float go[Q]) {
    const float om = p.omega, om1 = p.omega1;
    float mxx = om1 * m.mxx + om * m.ux * m.ux;
    float myy = om1 * m.myy + om * m.uy * m.uy;
    const float mxy = om1 * m.mxy + om * m.ux * m.uy;
    if (p.incomp_bulk) {
        const float t = 0.5f * (mxx + myy - m.ux * m.ux - m.uy * m.uy);
        mxx -= t;
        myy -= t;
    }
    const float A = 4.5f * mxx, B = 4.5f * myy, C = 9.0f * mxy;
    const float hm = p.hm, hp = p.hp;
    const float b0 = (A + B) * hm, bx = A * hp + B * hm, by = A * hm + B * hp, bd = (A + B) * hp;
    const float tx = 3.0f * m.ux, ty = 3.0f * m.uy, tp = 3.0f * (m.ux + m.uy), tm = 3.0f * (m.ux - m.uy);
    const float r = m.rho, d = m.drho;
    go[0] = p.w[0] * (d + r * b0);
    go[1] = p.w[1] * (d + r * (bx + tx));
    go[2] = p.w[1] * (d + r * (by + ty));
    go[3] = p.w[1] * (d + r * (bx - tx));
    go[4] = p.w[1] * (d + r * (by - ty));
    go[5] = p.w[5] * (d + r * ((bd + C) + tp));
    go[6] = p.w[5] * (d + r * ((bd - C) - tm));
    go[7] = p.w[5] * (d + r * ((bd + C) - tp));
    go[8] = p.w[5] * (d + r * ((bd - C) + tm));
}

// Velocity and rotated second moments of one bilinear stencil node (2d_mrlbm.f90:842-867).
__device__ __forceinline__ void stencil_node(const P& p, int si, int sj, float cc, float ss, float s2, float& ux,
                                             float& uy, float& mx, float& my) {
    float g[Q];
    gather(p, si, sj, g);
    const Mac m = moments(p, g);
    ux = m.ux;
    uy = m.uy;
    mx = m.mxx * cc + m.myy * ss + m.mxy * s2;
    my = m.mxx * ss + m.myy * cc - m.mxy * s2;
}

// The rotated closures in deviation form: numerical_boundary_cases_rotation (strong,
// 2d_mrlbm.f90:1635-1765), _weak (1767-1871) and _rhoeq (1873-1972).  With
// W = sum_{Is} w = sum_{Os} w (equal for every handled label), a_k = 3 w_k c'.u' and
// e_k = 4.5 w_k (u'u' : H'_k), the closures' O(1) parts cancel exactly:  rho_I = W + G and
// D_xy = SW_xy + d1 (d1 = sum_{Is} a_k H'xy_k); with gp the small part of the closure's
// reference sum (strong: G' = W + a1 + omega e2 over Os; weak: A' = W + a1 over Is; rho_eq:
// E' = W + a1 + e2 over Is),
//   R_xy = d1 - SG_xy - S_xy (gp - G) / rho_I   (rho_eq: its negative),
//   den  = W + dden,  drho = (G - dden) / den,
// dden = gp (+ (1 - omega) M'.B' strong, + M'.B' weak), B' summed where the closure sums it.
template <int VARIANT>
__device__ __forceinline__ void closure_rotated32(const P& p, const BTab<float>& tb, int li, const float g[Q], float uxp,
                                                  float uyp, float Mxx, float Myy, Mac& m) {
    const int Is = tb.gi(I_IS, li), Os = tb.gi(I_OS, li);
    const int label = tb.gi(I_LABEL, li);
    const float om = p.omega, om1 = p.omega1;
    float a1 = 0.f, e2 = 0.f, B11 = 0.f, B22 = 0.f, B12 = 0.f;
    float G = 0.f, SWxy = 0.f, SGxy = 0.f, d1 = 0.f, F11 = 0.f, F22 = 0.f, F12 = 0.f;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const float cxp = tb.gf(G_CXP + k, li), cyp = tb.gf(G_CYP + k, li);
        const float hxx = tb.gf(G_HXXP + k, li), hyy = tb.gf(G_HYYP + k, li), hxy = tb.gf(G_HXYP + k, li);
        const float wk = p.w[k];
        const float ak = 3.0f * wk * (uxp * cxp + uyp * cyp);
        const float ek = 4.5f * wk * ((uxp * uxp) * hxx + (uyp * uyp) * hyy + 2.0f * (uxp * uyp) * hxy);
        const float b11 = 4.5f * wk * hxx, b22 = 4.5f * wk * hyy, b12 = 4.5f * wk * hxy;
        const bool sum_here = VARIANT == CLOSURE_STRONG ? ((Os >> k) & 1) : ((Is >> k) & 1);
        if (sum_here) { a1 += ak; e2 += ek; B11 += b11; B22 += b22; B12 += b12; }
        if ((Is >> k) & 1) {
            G += g[k];
            SWxy += wk * hxy;
            SGxy += g[k] * hxy;
            d1 += ak * hxy;
            F11 += b11 * hxy;
            F22 += b22 * hxy;
            F12 += b12 * hxy;
        }
    }
    const float W = p.dc.lab_w[label];
    const float rhoI = W + G;
    const float Sxy = SWxy + SGxy;
    const float mxyI = Sxy / rhoI;
    float Mxy, dden;
    if constexpr (VARIANT == CLOSURE_STRONG) {
        const float L11 = om1 * B11 * mxyI - F11, L22 = om1 * B22 * mxyI - F22, L12 = 2.0f * (om1 * B12 * mxyI - F12);
        const float R = d1 - SGxy - Sxy * ((a1 + om * e2) - G) / rhoI;
        Mxy = (R - Mxx * L11 - Myy * L22) / L12;
        dden = a1 + om1 * (Mxx * B11 + Myy * B22 + 2.0f * Mxy * B12) + om * e2;
    } else if constexpr (VARIANT == CLOSURE_WEAK) {
        const float L11 = B11 * mxyI - F11, L22 = B22 * mxyI - F22, L12 = 2.0f * (B12 * mxyI - F12);
        const float R = d1 - SGxy - Sxy * (a1 - G) / rhoI;
        Mxy = (R - Mxx * L11 - Myy * L22) / L12;
        dden = a1 + (Mxx * B11 + Myy * B22 + 2.0f * Mxy * B12);
    } else {                                                // CLOSURE_RHOEQ
        const float R = SGxy - d1 + Sxy * ((a1 + e2) - G) / rhoI;
        Mxy = (R - Mxx * F11 - Myy * F22) / (2.0f * F12);
        dden = a1 + e2;
    }
    m.drho = (G - dden) / (W + dden);
    m.rho = 1.0f + m.drho;
    const float cc = tb.gf(G_CC, li), ss = tb.gf(G_SS, li), s2 = tb.gf(G_S2TH, li), c2 = tb.gf(G_C2TH, li);
    m.mxx = Mxx * cc + Myy * ss - Mxy * s2;
    m.myy = Mxx * ss + Myy * cc + Mxy * s2;
    m.mxy = (Mxx - Myy) * 0.5f * s2 + Mxy * c2;
}

// numerical_boundary_cases + solve_system (2d_mrlbm.f90:1496-1633, 1974-2003) in deviation
// form: the same 3 x 3 system for (Mxx, Myy, Mxy) by Cramer's rule, its coefficients O(1) and
// its right-hand side rearranged so the O(1) parts cancel exactly (S_ab = SW_ab + SG_ab,
// D_ab = SW_ab + d_ab, G' = W + gp with gp = a1 + omega e2 over Os):
//   rhs_ab = d_ab + (SW_ab (G - gp) - (W + gp) SG_ab) / rho_I,
// so a node at rest gives M = 0 exactly; drho = (G - dden) / (W + dden) with
// dden = gp + (1 - omega) M.B.
__device__ __forceinline__ void closure_unrotated32(const P& p, const BTab<float>& tb, int li, const float g[Q], float ux,
                                                    float uy, Mac& m) {
    const int Is = tb.gi(I_IS, li), Os = tb.gi(I_OS, li);
    const int label = tb.gi(I_LABEL, li);
    const float om = p.omega, om1 = p.omega1, hm = p.hm, hp = p.hp;
    float a1 = 0.f, e2 = 0.f, B11 = 0.f, B22 = 0.f, B12 = 0.f, G = 0.f;
    float SW[3] = {0.f, 0.f, 0.f}, SG[3] = {0.f, 0.f, 0.f}, dd[3] = {0.f, 0.f, 0.f};
    float F11[3] = {0.f, 0.f, 0.f}, F22[3] = {0.f, 0.f, 0.f}, F12[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const float h[3] = {hxx_of(k, hm, hp), hyy_of(k, hm, hp), (float)(ex(k) * ey(k))};
        const float wk = p.w[k];
        const float ak = 3.0f * wk * (ux * (float)ex(k) + uy * (float)ey(k));
        const float ek = 4.5f * wk * ((ux * ux) * h[0] + (uy * uy) * h[1] + 2.0f * (ux * uy) * h[2]);
        const float b11 = 4.5f * wk * h[0], b22 = 4.5f * wk * h[1], b12 = 4.5f * wk * h[2];
        if ((Os >> k) & 1) { a1 += ak; e2 += ek; B11 += b11; B22 += b22; B12 += b12; }
        if ((Is >> k) & 1) {
            G += g[k];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                SW[r] += wk * h[r];
                SG[r] += g[k] * h[r];
                dd[r] += ak * h[r];
                F11[r] += b11 * h[r];
                F22[r] += b22 * h[r];
                F12[r] += b12 * h[r];
            }
        }
    }
    const float W = p.dc.lab_w[label];
    const float rhoI = W + G;
    const float gp = a1 + om * e2;
    float A[3], Bc[3], C[3], D[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const float mI = (SW[r] + SG[r]) / rhoI;
        A[r] = om1 * B11 * mI - F11[r];
        Bc[r] = om1 * B22 * mI - F22[r];
        C[r] = 2.0f * (om1 * B12 * mI - F12[r]);
        D[r] = dd[r] + (SW[r] * (G - gp) - (W + gp) * SG[r]) / rhoI;
    }
    const float a1_ = A[0], b1 = Bc[0], c1 = C[0], a2 = A[1], b2 = Bc[1], c2 = C[1], a3 = A[2], b3 = Bc[2], c3 = C[2];
    const float d1 = D[0], d2 = D[1], d3 = D[2];
    const float denom = a3 * b2 * c1 - a2 * b3 * c1 - a3 * b1 * c2 + a1_ * b3 * c2 + a2 * b1 * c3 - a1_ * b2 * c3;
    const float Mxx = -((-b3 * c2 * d1 + b2 * c3 * d1 + b3 * c1 * d2 - b1 * c3 * d2 - b2 * c1 * d3 + b1 * c2 * d3) / denom);
    const float Myy = -((a3 * c2 * d1 - a2 * c3 * d1 - a3 * c1 * d2 + a1_ * c3 * d2 + a2 * c1 * d3 - a1_ * c2 * d3) / denom);
    const float Mxy = -((-a3 * b2 * d1 + a2 * b3 * d1 + a3 * b1 * d2 - a1_ * b3 * d2 - a2 * b1 * d3 + a1_ * b2 * d3) / denom);
    const float dden = gp + om1 * (Mxx * B11 + Myy * B22 + 2.0f * Mxy * B12);
    m.drho = (G - dden) / (W + dden);
    m.rho = 1.0f + m.drho;
    m.mxx = Mxx;
    m.myy = Myy;
    m.mxy = Mxy;
}

// The closures other than the default one, out of line: inlined, their registers would be
// reserved in every kernel that carries the wall path, the bulk tiles of one-launch steps
// included.  The populations travel by value.
struct Pops32 { float v[Q]; };
static __device__ __noinline__ Mac closure_other32(const P& p, const BTab<float>& tb, int li, Pops32 g, float ux, float uy,
                                                   float mxxp, float myyp, Mac m) {
    if (p.closure == CLOSURE_UNROTATED) {
        closure_unrotated32(p, tb, li, g.v, ux, uy, m);
    } else {
        const float c = tb.gf(G_CTH, li), s = tb.gf(G_STH, li);
        const float uxp = ux * c + uy * s, uyp = uy * c - ux * s;
        if (p.closure == CLOSURE_WEAK) closure_rotated32<CLOSURE_WEAK>(p, tb, li, g.v, uxp, uyp, mxxp, myyp, m);
        else closure_rotated32<CLOSURE_RHOEQ>(p, tb, li, g.v, uxp, uyp, mxxp, myyp, m);
    }
    return m;
}

// Lane 0 of a boundary node: extrapolation (wall value 0), closure, collision, store and
// the momentum-exchange force accumulated in FP64 from w_k + g_k (2d_mrlbm.f90:558-591).
template <bool FULL, bool PRE>
__device__ __forceinline__ void boundary_close(const P& p, const BTab<float>& tb, int li, int l, const float* gpre, float ux2,
                                            float uy2, float mx2, float my2, float ux3, float uy3, float mx3, float my3,
                                            double& Fx, double& Fy) {
    const int i = tb.gi(I_NODEI, li), j = tb.gi(I_NODEJ, li);
    float g[Q];
    if (PRE) {
#pragma unroll
        for (int k = 0; k < Q; ++k) g[k] = gpre[k];
    } else {
        gather(p, i, j, g);
    }
    Mac m = moments(p, g);
    float mxxp = 0.f, myyp = 0.f;
    const float t2 = tb.gf(G_T2, li), t3 = tb.gf(G_T3, li);
    const bool rotated = p.closure != CLOSURE_UNROTATED;
    if (!rotated || p.vel_interp) { m.ux = t2 * ux2 - t3 * ux3; m.uy = t2 * uy2 - t3 * uy3; }
    if (rotated && p.mom_interp) { mxxp = t2 * mx2 - t3 * mx3; myyp = t2 * my2 - t3 * my3; }
    if (p.closure == CLOSURE_STRONG) {
        const float c = tb.gf(G_CTH, li), s = tb.gf(G_STH, li);
        closure_rotated32<CLOSURE_STRONG>(p, tb, li, g, m.ux * c + m.uy * s, m.uy * c - m.ux * s, mxxp, myyp, m);
    } else if (p.closure != CLOSURE_NONE) {
        Pops32 gv;
#pragma unroll
        for (int k = 0; k < Q; ++k) gv.v[k] = g[k];
        m = closure_other32(p, tb, li, gv, m.ux, m.uy, mxxp, myyp, m);
    }
    if (!(m.rho > 0.0f)) flag_bad_density(p);
    if (FULL && p.macro) store_macro(p, i, j, 1.0 + (double)m.drho, m.ux, m.uy, m.mxx, m.myy, m.mxy);
    if (FULL && p.fstat) accumulate_fields(p, i, j, 1.0 + (double)m.drho, m.ux, m.uy);
    float go[Q];
    collide(p, m, go);
    store(p, i, j, go);
    const int Is = tb.gi(I_IS, li), Os = tb.gi(I_OS, li);
    double fxo = 0.0, fyo = 0.0, fxi = 0.0, fyi = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double wk = (double)p.w[k];
        if ((Os >> k) & 1) { const double v = wk + (double)go[k]; fxo += v * ex(k); fyo += v * ey(k); }
        if ((Is >> k) & 1) { const double v = wk + (double)g[k]; fxi += v * ex(k); fyi += v * ey(k); }
    }
    Fx = fxi - fxo;
    Fy = fyi - fyo;
    if (p.node_force) { p.node_force[2 * l] = Fx; p.node_force[2 * l + 1] = Fy; }
}

// Edge nodes: own gather, Dirichlet values and closures.  Inline, so the populations stay in
// registers and the gathers of a node overlap.
template <bool FULL>
__device__ __forceinline__ double edge_bulk_node(const P& p, int i, int j, int cls) {
    float g[Q];
    gather(p, i, j, g);
    Mac m = moments(p, g);
    edge_node(p, i, j, g, m);
    if ((cls == CLS_SOLID && p.zero_solid_u) || cls == CLS_SOLID_ZERO) { m.ux = 0.f; m.uy = 0.f; }
    if (!(m.rho > 0.0f)) flag_bad_density(p);
    if (FULL && p.macro) store_macro(p, i, j, 1.0 + (double)m.drho, m.ux, m.uy, m.mxx, m.myy, m.mxy);
    if (FULL && p.fstat) accumulate_fields(p, i, j, 1.0 + (double)m.drho, m.ux, m.uy);
    float go[Q];
    collide(p, m, go);
    if (FULL && p.body) add_body_force(p, i, j, go);
    store(p, i, j, go);
    return 1.0 + (double)m.drho;
}

// Interior fluid or solid node: populations already gathered.
template <bool FULL>
__device__ __forceinline__ void compute(const P& p, int i, int j, int cls, const float g[Q], float go[Q]) {
    FieldPre pre;
    if (FULL && p.fstat) fields_load(p, i, j, pre);
    Mac m = moments(p, g);
    if ((cls == CLS_SOLID && p.zero_solid_u) || cls == CLS_SOLID_ZERO) { m.ux = 0.f; m.uy = 0.f; }
    if (!(m.rho > 0.0f)) flag_bad_density(p);
    if (FULL && p.macro) store_macro(p, i, j, 1.0 + (double)m.drho, m.ux, m.uy, m.mxx, m.myy, m.mxy);
    if (FULL && p.fstat) fields_store(p, i, j, pre, 1.0 + (double)m.drho, m.ux, m.uy);
    collide(p, m, go);
    if (FULL && p.body) add_body_force(p, i, j, go);
}

template <bool FULL>
__device__ __forceinline__ void finish(const P& p, int i, int j, int cls, const float g[Q]) {
    float go[Q];
    compute<FULL>(p, i, j, cls, g, go);
    store(p, i, j, go);
}

// FULL: the node paths include the optional per-node work (field statistics, macroscopic
// output, body force), each behind its run-time switch.  The lean instantiation leaves it
// out; the launchers pick it when all three are off, which keeps the registers and the
// branches of that work out of the common step.
template <bool FULL>
struct PhysicsT {
    using P = StepParams<float>;
    using T = float;
    static __device__ __forceinline__ void compute(const P& p, int i, int j, int cls, const T f[Q], T fo[Q]) {
        fp32::compute<FULL>(p, i, j, cls, f, fo);
    }
    static __device__ __forceinline__ void finish(const P& p, int i, int j, int cls, const T g[Q]) {
        fp32::finish<FULL>(p, i, j, cls, g);
    }
    static __device__ __forceinline__ double edge_bulk_node(const P& p, int i, int j, int cls) {
        return fp32::edge_bulk_node<FULL>(p, i, j, cls);
    }
    static __device__ __forceinline__ void stencil_node(const P& p, int si, int sj, T cc, T ss, T s2, T& ux, T& uy,
                                                        T& mx, T& my) {
        fp32::stencil_node(p, si, sj, cc, ss, s2, ux, uy, mx, my);
    }
    static __device__ __forceinline__ void boundary_close(const P& p, const BTab<T>& tb, int li, int l, T ux2, T uy2,
                                                          T mx2, T my2, T ux3, T uy3, T mx3, T my3, double& Fx,
                                                          double& Fy) {
        fp32::boundary_close<FULL, false>(p, tb, li, l, nullptr, ux2, uy2, mx2, my2, ux3, uy3, mx3, my3, Fx, Fy);
    }
    static __device__ __forceinline__ void boundary_close_pre(const P& p, const BTab<T>& tb, int li, int l, const T g[Q],
                                                              T ux2, T uy2, T mx2, T my2, T ux3, T uy3, T mx3, T my3,
                                                              double& Fx, double& Fy) {
        fp32::boundary_close<FULL, true>(p, tb, li, l, g, ux2, uy2, mx2, my2, ux3, uy3, mx3, my3, Fx, Fy);
    }
    // registers per thread a kernel needs before its wall node's populations are gathered ahead
    static constexpr int WIDE_REGS = 96;
    // One launch per step with tile shapes: the FP32 wall closures fit the tiles' register
    // budgets, so the wall and edge blocks run as the first blocks of the bulk grid.
    static constexpr bool FUSED_AUX = true;
};
using Physics = PhysicsT<true>;
using PhysicsLean = PhysicsT<false>;

}  // namespace fp32
}  // namespace mrlbm
