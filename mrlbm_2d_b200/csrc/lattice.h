// lattice.h -- D2Q9 constants, the padded population layout and the streaming source rule,
// shared by host and device code.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define MRLBM_HD __host__ __device__ __forceinline__
#else
#define MRLBM_HD inline
#endif

namespace mrlbm {

constexpr int Q = 9;

// D2Q9 order of 2d_mrlbm.f90:130-131: 0 rest, 1 +x, 2 +y, 3 -x, 4 -y, 5 (+,+), 6 (-,+), 7 (-,-), 8 (+,-)
MRLBM_HD constexpr int ex(int k) { return (k == 1 || k == 5 || k == 8) ? 1 : ((k == 3 || k == 6 || k == 7) ? -1 : 0); }
MRLBM_HD constexpr int ey(int k) { return (k == 2 || k == 5 || k == 6) ? 1 : ((k == 4 || k == 7 || k == 8) ? -1 : 0); }
// y-mirror (specular reflection off a horizontal wall): 2<->4, 5<->8, 6<->7
MRLBM_HD constexpr int mirror_y(int k) {
    return k == 2 ? 4 : k == 4 ? 2 : k == 5 ? 8 : k == 8 ? 5 : k == 6 ? 7 : k == 7 ? 6 : k;
}

// Populations live in one buffer per time level, SoA by direction, i fastest (the
// reference's f(nx,ny,0:8) order) with a one-node ghost ring: node (i,j), i in 0..nx+1,
// j in 0..ny+1 (1-based interior), direction k sits at k*plane + j*pitch + i + off.
// `off` puts interior column 1 on a 128-byte boundary; pitch is a multiple of 32 elements.
// Ghost cells hold the populations the reference never overwrites at non-periodic edges
// (they keep their initial value, 2d_mrlbm.f90:509-517); kernels never write them.
struct Layout {
    int nx, ny;
    int pitch;        // elements per row (>= off + nx + 4: ghost column plus 128-bit read slack)
    int off;          // element offset of column 0
    int64_t plane;    // elements per direction plane = pitch * (ny + 2)
    MRLBM_HD int64_t at(int i, int j, int k) const { return (int64_t)k * plane + (int64_t)j * pitch + i + off; }
    MRLBM_HD int64_t total() const { return (int64_t)Q * plane; }
};

inline Layout make_layout(int nx, int ny, int align_elems) {
    Layout L;
    L.nx = nx;
    L.ny = ny;
    L.off = align_elems - 1;                                   // column 1 at index align_elems
    int need = L.off + nx + 4;                                 // 16-byte reads starting at i <= nx stay in the row
    L.pitch = ((need + align_elems - 1) / align_elems) * align_elems;
    L.plane = (int64_t)L.pitch * (ny + 2);
    return L;
}

// Streaming, pull form.  The reference pushes post-collision populations
// f(i+e_k, j+e_k, k) = fout(i,j,k) for in-domain targets (2d_mrlbm.f90:508-517), then
// applies its x-periodic wrap (same row, no diagonal shift; 2d_mrlbm.f90:519-526) and its
// y-periodic wrap (same column, no diagonal shift; 2d_mrlbm.f90:528-535), the later wrap
// winning.  Equivalently, f(i,j,k) at the next step is the fout value at the source slot
// this function returns.  Destinations nothing writes map to their own ghost slot
// (i-e_kx, j-e_ky, k) outside the interior, which keeps the population's initial value.
// Extension FREESLIP (only when !yper): populations leaving through rows 1/ny return
// specularly to the same row (source column wrapped when xper), applied after the wraps.
struct SrcSlot { int i, j, k; };

// For an x-slab of a larger domain (hl / hr: the left / right neighbour's populations sit in
// column 0 / nx+1), a reflection whose source column is that halo column reads it there.
MRLBM_HD SrcSlot stream_source(int nx, int ny, int i, int j, int k, bool xper, bool yper, bool freeslip,
                               bool hl = false, bool hr = false) {
    const int dx = ex(k), dy = ey(k);
    SrcSlot s{i - dx, j - dy, k};
    if (freeslip && !yper && ((j == ny && dy == -1) || (j == 1 && dy == 1))) {
        int ti = i - dx;
        if ((ti >= 1 || hl) && (ti <= nx || hr)) { s.i = ti; s.j = j; s.k = mirror_y(k); }
        else if (xper) { s.i = ti < 1 ? nx : 1; s.j = j; s.k = mirror_y(k); }
        return s;
    }
    if (yper && j == 1 && dy == 1) { s.i = i; s.j = ny; return s; }
    if (yper && j == ny && dy == -1) { s.i = i; s.j = 1; return s; }
    if (xper && i == 1 && dx == 1) { s.i = nx; s.j = j; return s; }
    if (xper && i == nx && dx == -1) { s.i = 1; s.j = j; return s; }
    return s;
}

// Node class inside the cylinder bounding box (values >= 0 are boundary-node indices).
constexpr int CLS_FLUID = -1;
constexpr int CLS_SOLID = -2;
constexpr int CLS_SOLID_ZERO = -3;   // a solid node of a replayed launch's plot step: u = 0 before collision

// Boundary condition variants of the curved wall (2d_mrlbm.f90:280-311).
enum Closure : int {
    CLOSURE_STRONG = 0,     // numerical_boundary_cases_rotation (2d_mrlbm.f90:1635)
    CLOSURE_RHOEQ = 1,      // numerical_boundary_cases_rotation_rhoeq (2d_mrlbm.f90:1873)
    CLOSURE_WEAK = 2,       // numerical_boundary_cases_rotation_weak (2d_mrlbm.f90:1767)
    CLOSURE_UNROTATED = 3,  // numerical_boundary_cases + solve_system (2d_mrlbm.f90:1496, 1974)
    CLOSURE_NONE = 4,       // rotated path with no mass-BC flag set: moments kept
};

// Per-boundary-node scalar table, field-major (field f of node l at f*nb + l).
enum GeoField : int {
    G_CTH = 0, G_STH, G_S2TH, G_C2TH, G_CC, G_SS,   // own node: cos, sin, sin2, cos2, cos^2, sin^2
    G_T1, G_T2, G_T3,                               // extrapolation weights (2d_mrlbm.f90:809-811)
    G_XD2, G_YD2, G_XD3, G_YD3, G_XD4, G_YD4,       // bilinear offsets of reference points 2..4
    G_CXP = 15,                                     // cx_p[9]  (2d_mrlbm.f90:188)
    G_CYP = G_CXP + 9,                              // cy_p[9]
    G_HXXP = G_CYP + 9,                             // Hxx_p[9]
    G_HYYP = G_HXXP + 9,                            // Hyy_p[9]
    G_HXYP = G_HYYP + 9,                            // Hxy_p[9]
    G_SCC = G_HXYP + 9,                             // stencil node m (0..7): cos^2
    G_SSS = G_SCC + 8,                              //                        sin^2
    G_SS2 = G_SSS + 8,                              //                        sin2
    G_NFIELDS = G_SS2 + 8
};
// Integer table, field-major: node i, node j, Is mask, Os mask, quadrant label, then 12
// stencil nodes (ref points 2,3,4 x 4 corners) as i and j.
enum IntField : int { I_NODEI = 0, I_NODEJ, I_IS, I_OS, I_LABEL, I_SI = 5, I_SJ = 5 + 12, I_NFIELDS = 5 + 24 };

}  // namespace mrlbm
