// adjoint.cuh -- discrete adjoint of the FP64 step for the gradient of time-averaged drag.
//
// State of step n: the post-collision field F^n (the buffer a step writes).  Step n maps
// F^{n-1} to F^n node by node: node x gathers its inputs g_x from F^{n-1} (pull streaming),
// and its local map C_x gives the nine outputs F^n(x, :).  With J = (1/T) sum_{n in window}
// D^n, D^n the net drag of step n (a function of the wall nodes' inputs and outputs), the
// adjoint field lambda^n = dJ/dF^n obeys
//     lambda^{n-1}(slot) = sum over the consumers x of the slot of (dC_x/dg_x)^T lambda^n(x)
//                          + w_n dD^n/dF^{n-1}(slot),      w_n = 1/T inside the window,
// and the parameter gradients collect (dC_x/dtheta)^T lambda^n(x).  One adjoint step is one
// launch with three kinds of blocks, each node's contribution added atomically to
// lambda^{n-1} at the slots it pulled (a slot can feed several nodes: stencils, the outlet
// copy, corner wraps):
//   * bulk nodes (fluid and solid, not edge nodes, not curved-wall nodes): reverse mode
//     written out by hand: reconstruction -> collision -> moments (adjoint_bulk_node);
//   * edge nodes (inlet column i = 1, outlet column i = nx, and with no-slip reference walls
//     rows 1 and ny): one thread per (node, input), the node's
//     local map evaluated on dual numbers carrying the derivative along that input, then
//     contracted with lambda^n (the transposed Jacobian column); the inlet's extra input is
//     u_in(j), whose column gives the inlet-profile gradient;
//   * curved-wall nodes: likewise, over the node's 9 own inputs and the 72 inputs of its 8
//     bilinear stencil nodes, with the drag contribution of the node in the same pass.
// The local maps below restate the FP64 step's arithmetic (step_fp64.cuh) for a generic
// scalar; they cover every closure of the FP64 step: the curved-wall closures (rotated
// strong, weak and rho_eq, unrotated with Cramer's rule, none) with or without velocity and
// moment extrapolation; inlet and outlet edge closures and no-slip
// reference walls, each in its apply_bc and apply_bc_incomp form; free-slip or y-periodic top
// and bottom; the incomp_bulk collision.
#pragma once
#include "adjoint.h"
#include "step_fp64.cuh"

namespace mrlbm {
namespace adj {

// Populations of node (i, j) as FP64 f: FP64 storage as is, FP32 storage holds f - w_k.
template <class T>
__device__ __forceinline__ double to_f(const StepParams<T>& p, int k, T v) {
    return sizeof(T) == 8 ? (double)v : (double)p.w[k] + (double)v;
}

template <class T>
__device__ __forceinline__ void gather_d(const StepParams<T>& p, int i, int j, double f[Q]) {
    T g[Q];
    gather(p, i, j, g);
#pragma unroll
    for (int k = 0; k < Q; ++k) f[k] = to_f(p, k, g[k]);
}

// ---- dual numbers (value, derivative along one input) -----------------------------------
struct Dual {
    double v, d;
    __device__ Dual() : v(0.0), d(0.0) {}
    __device__ Dual(double a) : v(a), d(0.0) {}
    __device__ Dual(double a, double b) : v(a), d(b) {}
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual operator+(Dual a, double b) { return Dual(a.v + b, a.d); }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return Dual(a + b.v, b.d); }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return Dual(a.v - b, a.d); }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return Dual(a - b.v, -b.d); }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return Dual(a.v * b, a.d * b); }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return Dual(a * b.v, a * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return Dual(a.v / b, a.d / b); }
__device__ __forceinline__ Dual operator/(double a, Dual b) {
    const double q = a / b.v;
    return Dual(q, -q * b.d / b.v);
}

template <class S>
struct MacS { S rho, ux, uy, mxx, myy, mxy; };

template <class S>
__device__ __forceinline__ MacS<S> moments_s(const S f[Q], double hm, double hp) {
    MacS<S> m;
    S r = f[0];
    for (int k = 1; k < Q; ++k) r = r + f[k];
    const S inv = 1.0 / r;
    const S sx = ((((f[1] - f[3]) + f[5]) - f[6]) - f[7]) + f[8];
    const S sy = ((((f[2] - f[4]) + f[5]) + f[6]) - f[7]) - f[8];
    S sxx = f[0] * hm, syy = f[0] * hm;
#pragma unroll
    for (int k = 1; k < Q; ++k) {
        sxx = sxx + f[k] * (ex(k) != 0 ? hp : hm);
        syy = syy + f[k] * (ey(k) != 0 ? hp : hm);
    }
    const S sxy = ((f[5] - f[6]) + f[7]) - f[8];
    m.rho = r;
    m.ux = sx * inv;
    m.uy = sy * inv;
    m.mxx = sxx * inv;
    m.myy = syy * inv;
    m.mxy = sxy * inv;
    return m;
}

// Collision (2d_mrlbm.f90:407-415, incomp_bulk 419-428) and Hermite reconstruction
// (2d_mrlbm.f90:445-457).
template <class P, class S>
__device__ __forceinline__ void collide_s(const P& p, const MacS<S>& m, S fo[Q]) {
    const double om = p.omega, om1 = p.omega1;
    S mxx = om1 * m.mxx + om * m.ux * m.ux;
    S myy = om1 * m.myy + om * m.uy * m.uy;
    const S mxy = om1 * m.mxy + om * m.ux * m.uy;
    if (p.incomp_bulk) {
        const S t = 0.5 * (((mxx + myy) - m.ux * m.ux) - m.uy * m.uy);
        mxx = mxx - t;
        myy = myy - t;
    }
    const S a = 4.5 * mxx, b = 4.5 * myy, c = 9.0 * mxy;
    const S am = a * p.hm, ap = a * p.hp, bm = b * p.hm, bp = b * p.hp;
    const S t1 = 3.0 * m.ux, t2 = 3.0 * m.uy, t5 = 3.0 * (m.ux + m.uy), t8 = 3.0 * (m.ux - m.uy);
    const S w0 = p.w[0] * m.rho, w1 = p.w[1] * m.rho, w5 = p.w[5] * m.rho;
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

// Sums over an incoming mask normalised by rho_I (apply_bc prologue, 2d_mrlbm.f90:1249-1269).
template <class S>
__device__ __forceinline__ void incoming_s(const S f[Q], int mask, double hm, double hp, S& rhoI, S& mxxI, S& myyI,
                                           S& mxyI) {
    S r = 0.0, a = 0.0, b = 0.0, c = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        if (!((mask >> k) & 1)) continue;
        r = r + f[k];
        a = a + f[k] * (ex(k) != 0 ? hp : hm);
        b = b + f[k] * (ey(k) != 0 ? hp : hm);
        const int hxy = ex(k) * ey(k);
        if (hxy > 0) c = c + f[k];
        if (hxy < 0) c = c - f[k];
    }
    rhoI = r;
    const S inv = 1.0 / r;
    mxxI = a * inv;
    myyI = b * inv;
    mxyI = c * inv;
}

// Domain-edge node (i, j): moments, Dirichlet values and the apply_bc / apply_bc_incomp closure
// (2d_mrlbm.f90:249-272, 1237-1494): inlet column i = 1, outlet column i = nx (fn: the inputs
// of node (nx - 1, j), whose moments it copies), and with no-slip reference walls rows 1 and
// ny, whose closure wins at the corners.
template <class P, class S>
__device__ __forceinline__ void edge_map(const P& p, int i, int j, const S f[Q], const S fn[Q], S uin, S fo[Q]) {
    const bool outlet = i == p.L.nx, inlet = i == 1;
    const bool top = p.walls_ref && j == p.L.ny, bottom = p.walls_ref && j == 1;
    const double hm = p.hm, hp = p.hp, om = p.omega;
    MacS<S> m = moments_s(f, hm, hp);
    if (outlet) {
        S r = fn[0];
        for (int k = 1; k < Q; ++k) r = r + fn[k];
        const S inv = 1.0 / r;
        m.rho = r;
        m.ux = (((((fn[1] - fn[3]) + fn[5]) - fn[6]) - fn[7]) + fn[8]) * inv;
        m.uy = (((((fn[2] - fn[4]) + fn[5]) + fn[6]) - fn[7]) - fn[8]) * inv;
    }
    if (inlet) {
        m.ux = uin;
        m.uy = S(p.vinlet);
    }
    S rhoI, mxxI, myyI, mxyI;
    if (top || bottom) {
        m.ux = S(0.0);
        m.uy = S(0.0);
        incoming_s(f, top ? fp64::M_TOP : fp64::M_BOTTOM, hm, hp, rhoI, mxxI, myyI, mxyI);
        if (!p.incomp_bc) {
            m.rho = 3.0 * rhoI * (4.0 + 3.0 * (1.0 - om) * myyI) / (9.0 + om);
            const S rp = m.rho;
            m.mxx = 6.0 * rhoI * mxxI / (5.0 * rp);
            m.myy = (rp + 9.0 * rhoI * myyI) / (6.0 * rp);
            m.mxy = 2.0 * rhoI * mxyI / rp;
        } else {
            m.rho = 6.0 * rhoI / 5.0;
            m.mxx = S(0.0);
            m.myy = S(0.0);
            m.mxy = 5.0 * mxyI / 3.0;
        }
    } else if (inlet) {
        incoming_s(f, fp64::M_INLET, hm, hp, rhoI, mxxI, myyI, mxyI);
        if (!p.incomp_bc) {
            m.rho = (4.0 * rhoI + 3.0 * rhoI * mxxI) / (3.0 - 3.0 * m.ux);
            const S rp = m.rho;
            m.mxx = (rp + 9.0 * rhoI * mxxI + 3.0 * rp * m.ux) / (6.0 * rp);
            m.myy = 6.0 * rhoI * myyI / (5.0 * rp);
            m.mxy = 2.0 * rhoI * mxyI / rp;
        } else {
            m.rho = 6.0 * rhoI / ((5.0 - 3.0 * m.ux) - 3.0 * (m.ux * m.ux));
            const S rp = m.rho;
            m.mxx = m.ux * m.ux;
            m.myy = S(0.0);
            m.mxy = 2.0 * rhoI * mxyI / rp;
        }
    } else if (outlet) {
        incoming_s(f, fp64::M_OUTLET, hm, hp, rhoI, mxxI, myyI, mxyI);
        const S rp = m.rho;
        if (!p.incomp_bc) {
            m.mxx = (rp + 9.0 * rhoI * mxxI - 3.0 * rp * m.ux) / (6.0 * rp);
            m.myy = 6.0 * rhoI * myyI / (5.0 * rp);
        } else {
            m.mxx = m.ux * m.ux;
            m.myy = m.uy * m.uy;
        }
        m.mxy = (6.0 * rhoI * mxyI - rp * m.uy) / (3.0 * rp);
    }
    collide_s(p, m, fo);
}

// Edge node e of the adjoint's enumeration: column 1 (j = 1..ny), column nx, then, with
// no-slip reference walls, rows 1 and ny without the corners.
template <class P>
__device__ __forceinline__ void edge_node_ij(const P& p, int e, int& i, int& j) {
    const int nx = p.L.nx, ny = p.L.ny;
    if (e < ny) { i = 1; j = e + 1; }
    else if (e < 2 * ny) { i = nx; j = e - ny + 1; }
    else {
        const int q = e - 2 * ny, nr = nx - 2;
        i = 2 + (q < nr ? q : q - nr);
        j = q < nr ? 1 : ny;
    }
}

template <class P>
__device__ __forceinline__ double gf(const P& p, int field, int l) { return (double)__ldg(p.bgeo + (int64_t)field * p.nb + l); }
template <class P>
__device__ __forceinline__ int gi(const P& p, int field, int l) { return __ldg(p.bint + (int64_t)field * p.nb + l); }

// Rotated velocity and second moments of one bilinear stencil node (2d_mrlbm.f90:842-867).
template <class P, class S>
__device__ __forceinline__ void stencil_quad(const P& p, int l, int s, const S f[Q], S& u, S& v, S& mx, S& my) {
    const MacS<S> m = moments_s(f, p.hm, p.hp);
    const double c2 = gf(p, G_SCC + s, l), s2q = gf(p, G_SSS + s, l), sn2 = gf(p, G_SS2 + s, l);
    u = m.ux;
    v = m.uy;
    mx = m.mxx * c2 + m.myy * s2q + m.mxy * sn2;
    my = m.mxx * s2q + m.myy * c2 - m.mxy * sn2;
}

// Rotated closures (2d_mrlbm.f90:1635-1765 strong, 1767-1871 weak, 1873-1972 rho_eq) of wall
// node l for a generic scalar, as closure_rotated_body in step_fp64.cuh: density and the
// rotated shear moment from the incoming populations, the extrapolated rotated normal moments
// Mxx, Myy, then the moments rotated back.
template <int variant, class P, class S>
__device__ __forceinline__ void closure_rotated_s(const P& p, int l, const S f[Q], S uxp, S uyp, S Mxx, S Myy, MacS<S>& m) {
    const int Is = gi(p, I_IS, l), Os = gi(p, I_OS, l);
    const double omega = p.omega;
    S rhoI = 0.0, mxyI = 0.0, A_p = 0.0, E_p = 0.0, D_xy = 0.0;
    double B11 = 0, B22 = 0, B12 = 0, F11 = 0, F22 = 0, F12 = 0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double cxp = gf(p, G_CXP + k, l), cyp = gf(p, G_CYP + k, l);
        const double hxx = gf(p, G_HXXP + k, l), hyy = gf(p, G_HYYP + k, l), hxy = gf(p, G_HXYP + k, l);
        const double wk = p.w[k];
        const S A_i = wk * (1.0 + 3.0 * uxp * cxp + 3.0 * uyp * cyp);
        const S E_i = wk * (1.0 + 3.0 * uxp * cxp + 3.0 * uyp * cyp + 4.5 * (uxp * uxp) * hxx + 4.5 * (uyp * uyp) * hyy +
                            9.0 * (uxp * uyp) * hxy);
        const double B11_i = 4.5 * wk * hxx, B22_i = 4.5 * wk * hyy, B12_i = 4.5 * wk * hxy;
        const bool o = (Os >> k) & 1, in = (Is >> k) & 1;
        if constexpr (variant == CLOSURE_STRONG) if (o) { A_p = A_p + A_i; E_p = E_p + E_i; B11 += B11_i; B22 += B22_i; B12 += B12_i; }
        if (in) {
            rhoI = rhoI + f[k];
            mxyI = mxyI + f[k] * hxy;
            if constexpr (variant == CLOSURE_WEAK) { A_p = A_p + A_i; B11 += B11_i; B22 += B22_i; B12 += B12_i; }
            if constexpr (variant == CLOSURE_RHOEQ) E_p = E_p + E_i;
            D_xy = D_xy + A_i * hxy;
            F11 += B11_i * hxy;
            F22 += B22_i * hxy;
            F12 += B12_i * hxy;
        }
    }
    mxyI = mxyI / rhoI;
    S Mxy;
    if constexpr (variant == CLOSURE_STRONG) {
        const S G_p = (1.0 - omega) * A_p + omega * E_p;
        const double J11 = (1.0 - omega) * B11, J22 = (1.0 - omega) * B22, J12 = (1.0 - omega) * B12;
        const S L11 = J11 * mxyI - F11, L22 = J22 * mxyI - F22, L12 = 2.0 * (J12 * mxyI - F12);
        const S R = D_xy - G_p * mxyI;
        Mxy = (R - Mxx * L11 - Myy * L22) / L12;
        const S den = (1.0 - omega) * A_p + (1.0 - omega) * (Mxx * B11 + Myy * B22 + 2.0 * Mxy * B12) + omega * E_p;
        m.rho = rhoI / den;
    } else if constexpr (variant == CLOSURE_WEAK) {
        const S L11 = B11 * mxyI - F11, L22 = B22 * mxyI - F22, L12 = 2.0 * (B12 * mxyI - F12);
        const S R = D_xy - A_p * mxyI;
        Mxy = (R - Mxx * L11 - Myy * L22) / L12;
        const S den = A_p + (Mxx * B11 + Myy * B22 + 2.0 * Mxy * B12);
        m.rho = rhoI / den;
    } else {                                               // CLOSURE_RHOEQ
        const S R = E_p * mxyI - D_xy;
        Mxy = (R - Mxx * F11 - Myy * F22) / (2.0 * F12);
        m.rho = rhoI / E_p;
    }
    const double cc = gf(p, G_CC, l), ss = gf(p, G_SS, l), s2 = gf(p, G_S2TH, l), c2 = gf(p, G_C2TH, l);
    m.mxx = Mxx * cc + Myy * ss - Mxy * s2;
    m.myy = Mxx * ss + Myy * cc + Mxy * s2;
    m.mxy = (Mxx - Myy) * 0.5 * s2 + Mxy * c2;
}

// Unrotated closure with Cramer's rule (2d_mrlbm.f90:1496-1633, 1974-2003) for a generic
// scalar, as closure_unrotated in step_fp64.cuh.
template <class P, class S>
__device__ __forceinline__ void closure_unrotated_s(const P& p, int l, const S f[Q], S ux, S uy, MacS<S>& m) {
    const int Is = gi(p, I_IS, l), Os = gi(p, I_OS, l);
    const double omega = p.omega, hm = p.hm, hp = p.hp;
    S rhoI = 0.0, mxxI = 0.0, myyI = 0.0, mxyI = 0.0, A_p = 0.0, E_p = 0.0, D_xx = 0.0, D_yy = 0.0, D_xy = 0.0;
    double B11 = 0, B22 = 0, B12 = 0, F11_xx = 0, F12_xx = 0, F22_xx = 0, F11_yy = 0, F12_yy = 0, F22_yy = 0;
    double F11_xy = 0, F12_xy = 0, F22_xy = 0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double hxx = ex(k) != 0 ? hp : hm, hyy = ey(k) != 0 ? hp : hm, hxy = (double)(ex(k) * ey(k));
        const double wk = p.w[k];
        const S A_i = wk * (1.0 + 3.0 * ux * (double)ex(k) + 3.0 * uy * (double)ey(k));
        const S E_i = wk * (1.0 + 3.0 * ux * (double)ex(k) + 3.0 * uy * (double)ey(k) + 4.5 * (ux * ux) * hxx +
                            4.5 * (uy * uy) * hyy + 9.0 * (ux * uy) * hxy);
        const double B11_i = 4.5 * wk * hxx, B22_i = 4.5 * wk * hyy, B12_i = 4.5 * wk * hxy;
        if ((Os >> k) & 1) { A_p = A_p + A_i; E_p = E_p + E_i; B11 += B11_i; B22 += B22_i; B12 += B12_i; }
        if ((Is >> k) & 1) {
            rhoI = rhoI + f[k];
            mxxI = mxxI + f[k] * hxx;
            myyI = myyI + f[k] * hyy;
            mxyI = mxyI + f[k] * hxy;
            D_xx = D_xx + A_i * hxx; D_yy = D_yy + A_i * hyy; D_xy = D_xy + A_i * hxy;
            F11_xx += B11_i * hxx; F22_xx += B22_i * hxx; F12_xx += B12_i * hxx;
            F11_yy += B11_i * hyy; F22_yy += B22_i * hyy; F12_yy += B12_i * hyy;
            F11_xy += B11_i * hxy; F22_xy += B22_i * hxy; F12_xy += B12_i * hxy;
        }
    }
    const S inv = 1.0 / rhoI;
    mxxI = mxxI * inv;
    myyI = myyI * inv;
    mxyI = mxyI * inv;
    const S G_p = (1.0 - omega) * A_p + omega * E_p;
    const double J11 = (1.0 - omega) * B11, J22 = (1.0 - omega) * B22, J12 = (1.0 - omega) * B12;
    const S a1 = J11 * mxxI - F11_xx, b1 = J22 * mxxI - F22_xx, c1 = 2.0 * (J12 * mxxI - F12_xx);
    const S a2 = J11 * myyI - F11_yy, b2 = J22 * myyI - F22_yy, c2 = 2.0 * (J12 * myyI - F12_yy);
    const S a3 = J11 * mxyI - F11_xy, b3 = J22 * mxyI - F22_xy, c3 = 2.0 * (J12 * mxyI - F12_xy);
    const S d1 = D_xx - G_p * mxxI, d2 = D_yy - G_p * myyI, d3 = D_xy - G_p * mxyI;
    const S denom = a3 * b2 * c1 - a2 * b3 * c1 - a3 * b1 * c2 + a1 * b3 * c2 + a2 * b1 * c3 - a1 * b2 * c3;
    const S Mxx = -((-b3 * c2 * d1 + b2 * c3 * d1 + b3 * c1 * d2 - b1 * c3 * d2 - b2 * c1 * d3 + b1 * c2 * d3) / denom);
    const S Myy = -((a3 * c2 * d1 - a2 * c3 * d1 - a3 * c1 * d2 + a1 * c3 * d2 + a2 * c1 * d3 - a1 * c2 * d3) / denom);
    const S Mxy = -((-a3 * b2 * d1 + a2 * b3 * d1 + a3 * b1 * d2 - a1 * b3 * d2 - a2 * b1 * d3 + a1 * b2 * d3) / denom);
    const S den = (1.0 - omega) * A_p + (1.0 - omega) * (Mxx * B11 + Myy * B22 + 2.0 * Mxy * B12) + omega * E_p;
    m.rho = rhoI / den;
    m.mxx = Mxx;
    m.myy = Myy;
    m.mxy = Mxy;
}

// Curved-wall node l from its own inputs f and its 8 stencil nodes' (u, v, mx, my): bilinear
// interpolation at reference points 2 and 3, extrapolation to the node, the closure the case
// selects, collision (2d_mrlbm.f90:294-311, 768-928, 1496-2003, 407-457; the order of
// boundary_close_core in step_fp64.cuh) and the node's drag term (2d_mrlbm.f90:558-591).
// The eight stencil nodes' u, v and rotated moments come as plain values (qd[kind][t]); the
// one stencil node s whose inputs carry the derivative (s < 0: none) comes as duals.  Each
// operand is formed where it is used, so no per-thread array of stencil duals exists.
template <int CL, class P, class S>
__device__ __forceinline__ void wall_map(const P& p, int l, const S f[Q], const double (*qd)[8], int s, S us, S vs,
                                         S mxs, S mys, S fo[Q], S& drag) {
    auto val = [&](int kind, int t) -> S {
        if (t == s) return kind == 0 ? us : kind == 1 ? vs : kind == 2 ? mxs : mys;
        return S(qd[kind][t]);
    };
    S u[2], v[2], mx[2], my[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const double xd = gf(p, r == 0 ? G_XD2 : G_XD3, l), yd = gf(p, r == 0 ? G_YD2 : G_YD3, l);
        S row_u[2], row_v[2], row_mx[2], row_my[2];
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
            const int s0 = 4 * r + 2 * rr;
            row_u[rr] = (1.0 - xd) * val(0, s0) + xd * val(0, s0 + 1);
            row_v[rr] = (1.0 - xd) * val(1, s0) + xd * val(1, s0 + 1);
            row_mx[rr] = (1.0 - xd) * val(2, s0) + xd * val(2, s0 + 1);
            row_my[rr] = (1.0 - xd) * val(3, s0) + xd * val(3, s0 + 1);
        }
        u[r] = (1.0 - yd) * row_u[0] + yd * row_u[1];
        v[r] = (1.0 - yd) * row_v[0] + yd * row_v[1];
        mx[r] = (1.0 - yd) * row_mx[0] + yd * row_mx[1];
        my[r] = (1.0 - yd) * row_my[0] + yd * row_my[1];
    }
    const double t2 = gf(p, G_T2, l), t3 = gf(p, G_T3, l);
    constexpr bool rotated = CL != CLOSURE_UNROTATED;
    // the node's own moments survive only where no closure or extrapolation replaces them
    MacS<S> m;
    if (CL == CLOSURE_NONE || (rotated && !p.vel_interp)) m = moments_s(f, p.hm, p.hp);
    if (!rotated || p.vel_interp) {
        m.ux = t2 * u[0] - t3 * u[1];
        m.uy = t2 * v[0] - t3 * v[1];
    }
    S Mxx = 0.0, Myy = 0.0;
    if (rotated && p.mom_interp) {
        Mxx = t2 * mx[0] - t3 * mx[1];
        Myy = t2 * my[0] - t3 * my[1];
    }
    if constexpr (CL == CLOSURE_UNROTATED) {
        closure_unrotated_s(p, l, f, m.ux, m.uy, m);
    } else if constexpr (CL != CLOSURE_NONE) {
        const double c = gf(p, G_CTH, l), sn = gf(p, G_STH, l);
        closure_rotated_s<CL>(p, l, f, m.ux * c + m.uy * sn, m.uy * c - m.ux * sn, Mxx, Myy, m);
    }
    collide_s(p, m, fo);
    const int Is = gi(p, I_IS, l), Os = gi(p, I_OS, l);
    S fxo = 0.0, fxi = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        if (ex(k) == 0) continue;
        if ((Os >> k) & 1) fxo = fxo + fo[k] * (double)ex(k);
        if ((Is >> k) & 1) fxi = fxi + f[k] * (double)ex(k);
    }
    drag = fxi - fxo;
}

// ---- kernels ------------------------------------------------------------------------------

// Add c to lambda^{n-1} at the slot node (i, j) pulled for direction k (ghost slots hold
// constants and take nothing).
template <class P>
__device__ __forceinline__ void scatter(const P& p, const AdjArgs& a, int i, int j, int k, double c) {
    const SrcSlot sl = stream_source(p.L.nx, p.L.ny, i, j, k, p.xper, p.yper, p.freeslip);
    if (sl.i < 1 || sl.i > p.L.nx || sl.j < 1 || sl.j > p.L.ny) return;
    atomicAdd(a.lam_out + p.L.at(sl.i, sl.j, sl.k), c);
}

template <class P>
__device__ __forceinline__ void body_grad(const P& p, const AdjArgs& a, int i, int j, const double lam[Q]) {
    if (!a.grad_body) return;
    const int64_t n = (int64_t)(i - 1) + (int64_t)p.L.nx * (j - 1), N = (int64_t)p.L.nx * p.L.ny;
    double gx = 0.0, gy = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        gx += 3.0 * p.w[k] * ex(k) * lam[k];
        gy += 3.0 * p.w[k] * ey(k) * lam[k];
    }
    a.grad_body[n] += gx;
    a.grad_body[N + n] += gy;
}

// Bulk node, reverse mode by hand.  Forward: rho = sum g, u = j / rho, m = Pi / rho,
// m' = (1 - w) m + w u u, fo_k = w_k rho A_k with A_k = 1 + 3 c.u + 4.5 m'_xx Hxx
// + 4.5 m'_yy Hyy + 9 m'_xy Hxy.  Every load the node needs (its inputs, lambda^n, the
// body-gradient sums) is issued before the first use, so a node waits for memory once.
template <class P>
__device__ __forceinline__ void adjoint_bulk(const P& p, const AdjArgs& a, int t) {
    const int nx = p.L.nx, ny = p.L.ny;
    if (t >= nx * ny) return;
    const int j = 1 + t / nx, i = t - (j - 1) * nx + 1;
    if (!p.xper && (i == 1 || i == nx)) return;            // edge columns: adjoint_edge
    if (p.walls_ref && (j == 1 || j == ny)) return;        // no-slip wall rows: adjoint_edge
    const int cls = node_class(p, i, j);
    if (cls >= 0) return;                                  // curved-wall node: adjoint_wall
    const int64_t own = p.L.at(i, j, 0), plane = p.L.plane;
    double g[Q], lam[Q];
    gather_d(p, i, j, g);
#pragma unroll
    for (int k = 0; k < Q; ++k) lam[k] = __ldcg(a.lam_in + own + k * plane);
    const int64_t n = (int64_t)(i - 1) + (int64_t)nx * (j - 1), N = (int64_t)nx * ny;
    const bool bg = p.body && a.grad_body;
    double gbx = 0.0, gby = 0.0;
    if (bg) {
        gbx = a.grad_body[n];
        gby = a.grad_body[N + n];
    }
#pragma unroll
    for (int k = 0; k < Q; ++k) a.lam_in[own + k * plane] = 0.0;   // read once: the buffer becomes step n-2's target
    const fp64::Mac m = fp64::moments(g, p.hm, p.hp);
    const bool u_zero = cls == CLS_SOLID && p.zero_solid_u;
    const double ux = u_zero ? 0.0 : m.ux, uy = u_zero ? 0.0 : m.uy;
    const double om = p.omega, om1 = p.omega1;
    double mxx = om1 * m.mxx + om * ux * ux, myy = om1 * m.myy + om * uy * uy;
    const double mxy = om1 * m.mxy + om * ux * uy;
    if (p.incomp_bulk) {                                   // m'' = m' - t I, t = (tr m' - |u|^2) / 2
        const double t = 0.5 * (((mxx + myy) - ux * ux) - uy * uy);
        mxx -= t;
        myy -= t;
    }
    double rb = 0.0, uxb = 0.0, uyb = 0.0, mxxb = 0.0, myyb = 0.0, mxyb = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double hxx = ex(k) != 0 ? p.hp : p.hm, hyy = ey(k) != 0 ? p.hp : p.hm, hxy = (double)(ex(k) * ey(k));
        const double A = 1.0 + 3.0 * (ex(k) * ux + ey(k) * uy) + 4.5 * mxx * hxx + 4.5 * myy * hyy + 9.0 * mxy * hxy;
        rb += lam[k] * p.w[k] * A;
        const double Ab = lam[k] * p.w[k] * m.rho;
        uxb += 3.0 * ex(k) * Ab;
        uyb += 3.0 * ey(k) * Ab;
        mxxb += 4.5 * hxx * Ab;
        myyb += 4.5 * hyy * Ab;
        mxyb += 9.0 * hxy * Ab;
    }
    if (p.incomp_bulk) {
        const double tb = -(mxxb + myyb);
        mxxb += 0.5 * tb;
        myyb += 0.5 * tb;
        uxb -= tb * ux;
        uyb -= tb * uy;
    }
    // collision: m' = (1 - w) m + w u u
    uxb += om * (2.0 * ux * mxxb + uy * mxyb);
    uyb += om * (2.0 * uy * myyb + ux * mxyb);
    mxxb *= om1;
    myyb *= om1;
    mxyb *= om1;
    if (u_zero) { uxb = 0.0; uyb = 0.0; }
    const double inv = 1.0 / m.rho;
    double mu[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double hxx = ex(k) != 0 ? p.hp : p.hm, hyy = ey(k) != 0 ? p.hp : p.hm, hxy = (double)(ex(k) * ey(k));
        mu[k] = rb + inv * (uxb * (ex(k) - m.ux) + uyb * (ey(k) - m.uy) + mxxb * (hxx - m.mxx) + myyb * (hyy - m.myy) +
                            mxyb * (hxy - m.mxy));
    }
    const bool shared = i == nx - 1 || (i >= a.sx0 && i <= a.sx1 && j >= a.sy0 && j <= a.sy1);
    if (!shared && is_interior(p, i, j)) {
        // the nine source slots are this node's alone: plain stores into the zeroed buffer
        double* d = a.lam_out + own;
#pragma unroll
        for (int k = 0; k < Q; ++k) d[k * plane - ey(k) * (int64_t)p.L.pitch - ex(k)] = mu[k];
    } else {
#pragma unroll
        for (int k = 0; k < Q; ++k) scatter(p, a, i, j, k, mu[k]);
    }
    if (bg) {
        double gx = 0.0, gy = 0.0;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            gx += 3.0 * p.w[k] * ex(k) * lam[k];
            gy += 3.0 * p.w[k] * ey(k) * lam[k];
        }
        a.grad_body[n] = gbx + gx;
        a.grad_body[N + n] = gby + gy;
    }
}

// Edge nodes: thread (e, q), e over the n_edge nodes of edge_node_ij, q over 18 inputs: own
// inputs 0..8; at the outlet the copied neighbour's inputs 9..17; at the inlet q = 9 is u_in(j).
template <class P>
__device__ __forceinline__ void adjoint_edge(const P& p, const AdjArgs& a, int e, int q, const double* lam) {
    if (e >= a.n_edge) return;
    const int nx = p.L.nx;
    int i, j;
    edge_node_ij(p, e, i, j);
    const bool inlet = i == 1, outlet = i == nx;
    if (q > 9 && !outlet) return;
    if (q == 9 && !outlet && !inlet) return;
    double g[Q], gn[Q];
    gather_d(p, i, j, g);
    if (outlet) gather_d(p, nx - 1, j, gn);
    Dual f[Q], fn[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        f[k] = Dual(g[k], q == k ? 1.0 : 0.0);
        fn[k] = Dual(outlet ? gn[k] : 0.0, (outlet && q == 9 + k) ? 1.0 : 0.0);
    }
    const double u0 = p.u_in ? (double)p.u_in[j - 1] : (double)p.uinlet;
    const Dual uin(u0, (inlet && q == 9) ? 1.0 : 0.0);
    Dual fo[Q];
    edge_map(p, i, j, f, fn, uin, fo);
    double c = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) c += lam[k] * fo[k].d;
    if (q < 9) scatter(p, a, i, j, q, c);
    else if (outlet) scatter(p, a, nx - 1, j, q - 9, c);
    else if (a.grad_uin) a.grad_uin[j - 1] += c;
    if (q == 0 && p.body) body_grad(p, a, i, j, lam);
}

// Curved-wall node l, one block: the block stages the node's 81 inputs (9 own, 9 for each of
// its 8 stencil nodes) and the stencil quantities in shared memory; thread q < 81 then runs
// the node's map with the derivative along input q (only its stencil node's quantities carry
// a derivative) and scatters the contracted column.
template <int CL, class P>
__device__ __forceinline__ void adjoint_wall(const P& p, const AdjArgs& a, int l) {
    __shared__ double in[81], lam[Q], qd[4][8];
    __shared__ int slot[81];
    const int q = threadIdx.x;
    const int i = gi(p, I_NODEI, l), j = gi(p, I_NODEJ, l);
    if (q < 81) {
        int ni = i, nj = j, k = q;
        if (q >= 9) {
            const int s = (q - 9) / Q;
            ni = gi(p, I_SI + s, l);
            nj = gi(p, I_SJ + s, l);
            k = (q - 9) % Q;
        }
        const SrcSlot sl = stream_source(p.L.nx, p.L.ny, ni, nj, k, p.xper, p.yper, p.freeslip);
        const int64_t at = p.L.at(sl.i, sl.j, sl.k);
        in[q] = to_f(p, k, __ldg(p.src + at));
        const bool ghost = sl.i < 1 || sl.i > p.L.nx || sl.j < 1 || sl.j > p.L.ny;
        slot[q] = ghost ? -1 : (int)at;
    } else if (q < 81 + Q) {
        const int64_t at = p.L.at(i, j, q - 81);
        lam[q - 81] = a.lam_in[at];
        a.lam_in[at] = 0.0;                      // read once, into shared memory
    }
    __syncthreads();
    if (q < 8) {
        double f[Q], u, v, mx, my;
#pragma unroll
        for (int k = 0; k < Q; ++k) f[k] = in[9 + Q * q + k];
        stencil_quad(p, l, q, f, u, v, mx, my);
        qd[0][q] = u; qd[1][q] = v; qd[2][q] = mx; qd[3][q] = my;
    }
    __syncthreads();
    if (q >= 81) return;
    Dual f[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) f[k] = Dual(in[k], q == k ? 1.0 : 0.0);
    int s = -1;                                          // the stencil node input q belongs to
    Dual us(0.0), vs(0.0), mxs(0.0), mys(0.0);
    if (q >= 9) {
        s = (q - 9) / Q;
        const int kk = (q - 9) % Q;
        Dual g[Q];
#pragma unroll
        for (int k = 0; k < Q; ++k) g[k] = Dual(in[9 + Q * s + k], k == kk ? 1.0 : 0.0);
        stencil_quad(p, l, s, g, us, vs, mxs, mys);    // only stencil s depends on input q
    }
    Dual fo[Q], drag;
    wall_map<CL>(p, l, f, qd, s, us, vs, mxs, mys, fo, drag);
    double c = a.wJ * drag.d;
#pragma unroll
    for (int k = 0; k < Q; ++k) c += lam[k] * fo[k].d;
    if (slot[q] >= 0) atomicAdd(a.lam_out + slot[q], c);
}

// One adjoint step as two launches, ordered like the forward step's (step_common.cuh): the
// wall and edge blocks [nb wall blocks][edge blocks, 7 nodes x 18 inputs each], whose dual-number
// maps get the registers they need, then the bulk blocks (128 nodes each), which start once the
// first launch has waited for the previous step and run beside it; the last bulk block to finish
// waits for the first launch, so the step completes as a whole.
template <class P, int CL>
__global__ void __launch_bounds__(128) adjoint_aux(const __grid_constant__ P p, const __grid_constant__ AdjArgs a) {
    wait_prior_grid();
    const int b = (int)blockIdx.x;
    if (b < p.nb) {
        adjoint_wall<CL>(p, a, b);
        return;
    }
    // lambda^n of the block's 7 edge nodes, staged once and cleared for reuse
    __shared__ double lam[7][Q];
    const int t = threadIdx.x, e0 = 7 * (b - p.nb);
    if (t < 7 * Q) {
        const int e = e0 + t / Q, k = t % Q;
        if (e < a.n_edge) {
            int i, j;
            edge_node_ij(p, e, i, j);
            const int64_t at = p.L.at(i, j, k);
            lam[t / Q][k] = a.lam_in[at];
            a.lam_in[at] = 0.0;
        }
    }
    __syncthreads();
    if (t < 126) adjoint_edge(p, a, e0 + t / 18, t % 18, lam[t / 18]);
}

template <class P>
__global__ void __launch_bounds__(128, 4) adjoint_bulk_step(const __grid_constant__ P p, const __grid_constant__ AdjArgs a) {
    bulk_begin();
    adjoint_bulk(p, a, (int)blockIdx.x * 128 + (int)threadIdx.x);
    if (threadIdx.x == 0 && atomicAdd(a.done, 1u) == gridDim.x - 1) {
        *a.done = 0u;
        asm volatile("griddepcontrol.wait;" ::: "memory");
    }
}

}  // namespace adj
}  // namespace mrlbm
