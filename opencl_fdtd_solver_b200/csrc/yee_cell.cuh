// Per-cell Yee/CPML arithmetic shared by the split half-step kernels and the
// fused single-pass step kernel.
//
// The operation order of every expression follows the reference kernels
// (opencl_fdtd_solver/kernels/yee_update.cl) so that, compiled with
// --fmad=false, each cell rounds exactly as the reference's FP32/FP64 kernels
// do when every operation is rounded separately:
//   interior H  yee_update.cl:30-39   (folded dt/(mu0*dl))
//   CPML H      yee_update.cl:75-117  (kappa via 1/(kappa*dl), psi recursion)
//   interior E  yee_update.cl:145-154 (ce * (1/dl))
//   CPML E      yee_update.cl:195-237
//   sheet src   sources.cl:14-20, 36-48 (applied to E^n before the update)
#pragma once
#include <cstdint>
#include "../../include/fdtd_b200.h"

namespace fdtd {

template <typename T>
struct Cpml1D {
    const T *b[3], *c[3], *ik[3];
};

// ψ stripe offsets for one cell.  Layer l of axis a: low face l in [0,npml),
// high face npml + (x - (N - npml)) (yee_update.cl:91,99,107).  The x axis of
// a slab of an x-decomposed grid has lo low and hi high layers (npml on a
// global face, 0 on a face towards another slab); y and z have npml on both.
__device__ __forceinline__ int pml_layer(int x, int n, int lo, int hi) {
    return (x < lo) ? x : (lo + x - (n - hi));
}
__device__ __forceinline__ int pml_layer(int x, int n, int npml) {
    return pml_layer(x, n, npml, npml);
}

__device__ __forceinline__ bool in_slab(int x, int n, int lo, int hi) {
    return x < lo || x >= n - hi;
}
__device__ __forceinline__ bool in_slab(int x, int n, int npml) {
    return npml > 0 && (x < npml || x >= n - npml);
}

// The x range [xlo, nx - xhi) of interior cells: the x CPML layers are
// excluded and, on a slab, the ghost plane whose interior update would read
// past the slab (the upper ghost for H, the lower for E), which takes the
// boundary-guarded form instead.
__device__ __forceinline__ bool is_interior(int i, int j, int k, int nx, int ny, int nz,
                                            int npml, int xlo, int xhi) {
    return npml > 0 && i >= xlo && i < nx - xhi && j >= npml && j < ny - npml &&
           k >= npml && k < nz - npml;
}
__device__ __forceinline__ bool is_interior(int i, int j, int k, int nx, int ny, int nz,
                                            int npml) {
    return is_interior(i, j, k, nx, ny, nz, npml, npml, npml);
}

__device__ __forceinline__ int64_t psi_x_index(int i, int j, int k, int nx, int ny, int nz,
                                               int lo, int hi) {
    return ((int64_t)pml_layer(i, nx, lo, hi) * ny + j) * nz + k;
}
__device__ __forceinline__ int64_t psi_x_index(int i, int j, int k, int nx, int ny, int nz,
                                               int npml) {
    return psi_x_index(i, j, k, nx, ny, nz, npml, npml);
}

// x-CPML layers of a Yee kernel's grid: (lo, hi), and the interior x bounds.
struct XBounds {
    int pml_lo, pml_hi;  // x CPML layers at the low / high x face
    int h_lo, h_hi;      // interior H cells: x in [h_lo, nx - h_hi)
    int e_lo, e_hi;      // interior E cells: x in [e_lo, nx - e_hi)
};
__device__ __forceinline__ int64_t psi_y_index(int i, int j, int k, int ny, int nz, int npml) {
    return ((int64_t)i * (2 * npml) + pml_layer(j, ny, npml)) * nz + k;
}
__device__ __forceinline__ int64_t psi_z_index(int i, int j, int k, int ny, int nz, int npml) {
    return ((int64_t)i * ny + j) * (2 * npml) + pml_layer(k, nz, npml);
}

// Forward differences of E for one H cell: (dEz_dy, dEy_dz, dEx_dz, dEz_dx, dEy_dx, dEx_dy).
template <typename T>
struct DE {
    T zy, yz, xz, zx, yx, xy;
};

// H update of one cell given E differences (already zeroed at the high edges
// where the reference guards them) and the H values at the cell.
// psi_* point at the ψ_H stripes to read (rd) and write (wr); rd == wr for the
// in-place split kernel.  Returns the new H through hx/hy/hz.
template <typename T, bool WRITE_PSI = true>
__device__ __forceinline__ void h_cell(bool interior, int i, int j, int k, int nx, int ny,
                                       int nz, int npml, const XBounds &xb, T dtm, T dtm_dl,
                                       const DE<T> &d,
                                       const Cpml1D<T> &cp, T *const *psi_rd, T *const *psi_wr,
                                       T &hx, T &hy, T &hz) {
    if (interior) {
        hx = hx - dtm_dl * (d.zy - d.yz);
        hy = hy - dtm_dl * (d.xz - d.zx);
        hz = hz - dtm_dl * (d.yx - d.xy);
        return;
    }
    // psi order: 0 Hx_y, 1 Hx_z, 2 Hy_x, 3 Hy_z, 4 Hz_x, 5 Hz_y
    T p_hx_y = T(0), p_hx_z = T(0), p_hy_x = T(0), p_hy_z = T(0), p_hz_x = T(0), p_hz_y = T(0);
    if (npml > 0 && in_slab(i, nx, xb.pml_lo, xb.pml_hi)) {
        const int64_t s = psi_x_index(i, j, k, nx, ny, nz, xb.pml_lo, xb.pml_hi);
        const T b = cp.b[0][i], c = cp.c[0][i];
        p_hy_x = b * psi_rd[2][s] + c * d.zx;
        p_hz_x = b * psi_rd[4][s] + c * d.yx;
        if (WRITE_PSI) {
            psi_wr[2][s] = p_hy_x;
            psi_wr[4][s] = p_hz_x;
        }
    }
    if (in_slab(j, ny, npml)) {
        const int64_t s = psi_y_index(i, j, k, ny, nz, npml);
        const T b = cp.b[1][j], c = cp.c[1][j];
        p_hx_y = b * psi_rd[0][s] + c * d.zy;
        p_hz_y = b * psi_rd[5][s] + c * d.xy;
        if (WRITE_PSI) {
            psi_wr[0][s] = p_hx_y;
            psi_wr[5][s] = p_hz_y;
        }
    }
    if (in_slab(k, nz, npml)) {
        const int64_t s = psi_z_index(i, j, k, ny, nz, npml);
        const T b = cp.b[2][k], c = cp.c[2][k];
        p_hx_z = b * psi_rd[1][s] + c * d.yz;
        p_hy_z = b * psi_rd[3][s] + c * d.xz;
        if (WRITE_PSI) {
            psi_wr[1][s] = p_hx_z;
            psi_wr[3][s] = p_hy_z;
        }
    }
    const T ikx = cp.ik[0][i], iky = cp.ik[1][j], ikz = cp.ik[2][k];
    hx = hx - dtm * (d.zy * iky + p_hx_y - d.yz * ikz - p_hx_z);
    hy = hy - dtm * (d.xz * ikz + p_hy_z - d.zx * ikx - p_hy_x);
    hz = hz - dtm * (d.yx * ikx + p_hz_x - d.xy * iky - p_hz_y);
}

// Backward differences of H for one E cell: (dHz_dy, dHy_dz, dHx_dz, dHz_dx, dHy_dx, dHx_dy).
template <typename T>
struct DH {
    T zy, yz, xz, zx, yx, xy;
};

// Interior E update (yee_update.cl:145-154): folded ce * (1/dl).
template <typename T, bool LOSSY>
__device__ __forceinline__ void e_interior(const DH<T> &d, T inv_dl, T cax, T cay, T caz, T cex,
                                           T cey, T cez, T &ex, T &ey, T &ez) {
    ex = (LOSSY ? cax * ex : ex) + cex * inv_dl * (d.zy - d.yz);
    ey = (LOSSY ? cay * ey : ey) + cey * inv_dl * (d.xz - d.zx);
    ez = (LOSSY ? caz * ez : ez) + cez * inv_dl * (d.yx - d.xy);
}

// CPML E update given the six ψ_E terms of the cell (zero on the axes whose
// slab the cell is not in) and the 1/(kappa*dl) of its three coordinates
// (yee_update.cl:233-237).
template <typename T, bool LOSSY>
__device__ __forceinline__ void e_combine(const DH<T> &d, T ikx, T iky, T ikz, T p_ex_y,
                                          T p_ex_z, T p_ey_x, T p_ey_z, T p_ez_x, T p_ez_y,
                                          T cax, T cay, T caz, T cex, T cey, T cez, T &ex,
                                          T &ey, T &ez) {
    ex = (LOSSY ? cax * ex : ex) + cex * (d.zy * iky + p_ex_y - d.yz * ikz - p_ex_z);
    ey = (LOSSY ? cay * ey : ey) + cey * (d.xz * ikz + p_ey_z - d.zx * ikx - p_ey_x);
    ez = (LOSSY ? caz * ez : ez) + cez * (d.yx * ikx + p_ez_x - d.xy * iky - p_ez_y);
}

// E update of one cell.  ex/ey/ez enter as E^n (with any sheet injection
// already added) and leave as E^{n+1}.  psi_e is updated in place.
template <typename T, bool LOSSY>
__device__ __forceinline__ void e_cell(bool interior, int i, int j, int k, int nx, int ny,
                                       int nz, int npml, const XBounds &xb, T inv_dl,
                                       const DH<T> &d,
                                       const Cpml1D<T> &cp, T *const *psi_e, T cax, T cay,
                                       T caz, T cex, T cey, T cez, T &ex, T &ey, T &ez) {
    if (interior) {
        e_interior<T, LOSSY>(d, inv_dl, cax, cay, caz, cex, cey, cez, ex, ey, ez);
        return;
    }
    // psi order: 0 Ex_y, 1 Ex_z, 2 Ey_x, 3 Ey_z, 4 Ez_x, 5 Ez_y
    T p_ex_y = T(0), p_ex_z = T(0), p_ey_x = T(0), p_ey_z = T(0), p_ez_x = T(0), p_ez_y = T(0);
    if (npml > 0 && in_slab(i, nx, xb.pml_lo, xb.pml_hi)) {
        const int64_t s = psi_x_index(i, j, k, nx, ny, nz, xb.pml_lo, xb.pml_hi);
        const T b = cp.b[0][i], c = cp.c[0][i];
        p_ey_x = b * psi_e[2][s] + c * d.zx;
        p_ez_x = b * psi_e[4][s] + c * d.yx;
        psi_e[2][s] = p_ey_x;
        psi_e[4][s] = p_ez_x;
    }
    if (in_slab(j, ny, npml)) {
        const int64_t s = psi_y_index(i, j, k, ny, nz, npml);
        const T b = cp.b[1][j], c = cp.c[1][j];
        p_ex_y = b * psi_e[0][s] + c * d.zy;
        p_ez_y = b * psi_e[5][s] + c * d.xy;
        psi_e[0][s] = p_ex_y;
        psi_e[5][s] = p_ez_y;
    }
    if (in_slab(k, nz, npml)) {
        const int64_t s = psi_z_index(i, j, k, ny, nz, npml);
        const T b = cp.b[2][k], c = cp.c[2][k];
        p_ex_z = b * psi_e[1][s] + c * d.yz;
        p_ey_z = b * psi_e[3][s] + c * d.xz;
        psi_e[1][s] = p_ex_z;
        psi_e[3][s] = p_ey_z;
    }
    e_combine<T, LOSSY>(d, cp.ik[0][i], cp.ik[1][j], cp.ik[2][k], p_ex_y, p_ex_z, p_ey_x, p_ey_z,
                        p_ez_x, p_ez_y, cax, cay, caz, cex, cey, cez, ex, ey, ez);
}

// Pending sheet injections for one launch, passed by value.
struct SourceList {
    fdtd_source s[FDTD_MAX_SOURCES];
    int n;
};

// Apply the injections that hit cell (i, j, k) to E^n of Ex, in list order.
template <typename T>
__device__ __forceinline__ T apply_sources(const SourceList &sl, int i, int j, int k, T ex,
                                           T cex) {
    for (int q = 0; q < sl.n; ++q) {
        const fdtd_source &s = sl.s[q];
        if (k != s.z || i < s.i0 || i >= s.i1 || j < s.j0 || j >= s.j1) continue;
        const T amp = (T)s.amp;
        if (s.kind == FDTD_SRC_EX) {
            ex = ex + amp;
        } else {
            T w = T(1);
            if (s.rim_taper) {
                const T re = (T)s.rim_edge;
                if (i == s.i0 || i == s.i1 - 1) w = w * re;
                if (j == s.j0 || j == s.j1 - 1) w = w * re;
            }
            ex = ex + -cex * amp * w;
        }
    }
    return ex;
}

// Fused plane DFT descriptors, passed by value.
struct PlaneList {
    fdtd_plane_dft p[FDTD_MAX_PLANES];
    int n;
};

// True when cell (i, j, k) lies on one of the DFT planes (integer tests only,
// so the per-cell cost away from the planes is a few compares).
__device__ __forceinline__ bool plane_any_hit(const PlaneList &pl, int i, int j, int k) {
    bool hit = false;
    for (int q = 0; q < pl.n; ++q) {
        const fdtd_plane_dft &p = pl.p[q];
        hit |= (p.axis == 0) ? (i == p.index) : (p.axis == 1) ? (j == p.index) : (k == p.index);
    }
    return hit;
}

// Accumulate the plane DFTs that contain cell (i, j, k).  v[0..5] are the
// cell's Ex, Ey, Ez (at step n+1) and Hx, Hy, Hz (at n+1/2).
__device__ __forceinline__ void plane_dft_cell(const PlaneList &pl, int i, int j, int k, int nx,
                                               int ny, int nz, const double v[6]) {
    for (int q = 0; q < pl.n; ++q) {
        const fdtd_plane_dft &p = pl.p[q];
        int64_t cell, ncell;
        if (p.axis == 0) {
            if (i != p.index) continue;
            cell = (int64_t)j * nz + k;
            ncell = (int64_t)ny * nz;
        } else if (p.axis == 1) {
            if (j != p.index) continue;
            cell = (int64_t)i * nz + k;
            ncell = (int64_t)nx * nz;
        } else {
            if (k != p.index) continue;
            cell = (int64_t)i * ny + j;
            ncell = (int64_t)nx * ny;
        }
        int slot = 0;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            if (!(p.comp_mask & (1 << c))) continue;
            const int h = c >= 3 ? 2 : 0;
            for (int f = 0; f < p.nfreq; ++f) {
                const double pr = p.phase[4 * f + h], pi = p.phase[4 * f + h + 1];
                double2 *a = reinterpret_cast<double2 *>(p.acc) + ((int64_t)slot * p.nfreq + f) * ncell + cell;
                double2 cur = *a;
                cur.x = cur.x + v[c] * pr;
                cur.y = cur.y + v[c] * pi;
                *a = cur;
            }
            ++slot;
        }
    }
}

// The plane DFTs of one cell, called out of line from the shell kernels.
// planes points at the kernel's __grid_constant__ parameter, so the call takes
// no local copy of the descriptor list.
static __device__ __noinline__ void shell_dft(const PlaneList *planes, int i, int j, int k,
                                              int nx, int ny, int nz, double ex, double ey,
                                              double ez, double hx, double hy, double hz) {
    const double v[6] = {ex, ey, ez, hx, hy, hz};
    plane_dft_cell(*planes, i, j, k, nx, ny, nz, v);
}

}  // namespace fdtd
