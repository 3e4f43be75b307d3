// CPML shell half-steps of the fused schedule.
//
// The fused step splits the grid into the interior box handled by the
// single-pass kernel (yee_fused.cu) and a shell around it handled here, one
// thread per cell:
//   k_shell_H : H^{n+1/2} of every cell outside the box B = [lo, hi)^3 (the
//               CPML slabs; the whole grid when there is no box), H read from H
//               and written to H_next, psi_H in place.
//   k_shell_E : E^{n+1} of the cells of an outer box that lie outside an inner
//               box, reading H^{n+1/2} from H_next, writing E_next, psi_E in
//               place, with the sheet injections and plane DFTs of those cells.
//               The fused step launches it twice: for the cells outside
//               [lo, hi+1)^3, whose stencils read no H of B (right after
//               k_shell_H, concurrent with the interior kernel), and for the
//               one-cell rim [lo, hi+1)^3 minus [lo+1, hi)^3, whose stencils do
//               (after the interior kernel).
// Per-cell arithmetic is yee_cell.cuh (reference yee_update.cl), so each cell
// rounds exactly as in the split kernels.
//
// Shell enumeration: a flat cell index over three disjoint groups of the outer
// box o minus the inner box b,
//   A: i in o, outside b                          all (j, k) of o
//   B: i in b, j in o outside b                   all k of o
//   C: i in b, j in b, k in o outside b
// decoded with multiply-high divisions (consecutive threads take consecutive k).
#include <cuda_runtime.h>

#include "launch_count.cuh"
#include "shell_plan.cuh"
#include "yee_launch.cuh"

namespace fdtd {


template <typename T>
__global__ void __launch_bounds__(SHELL_THREADS)
    k_shell_H(YeeArgs<T> a, ShellPlan sp) {
    const int nx = a.nx, ny = a.ny, nz = a.nz, npml = a.npml;
    int i, j, k;
    if (!shell_cell(blockIdx.x * SHELL_THREADS + threadIdx.x, sp, i, j, k)) return;
    const int64_t sx = (int64_t)ny * nz, sy = nz;
    const int64_t idx = (int64_t)i * sx + (int64_t)j * sy + k;
    const T *Ex = a.E[0], *Ey = a.E[1], *Ez = a.E[2];
    const bool interior =
        is_interior(i, j, k, nx, ny, nz, npml, a.xb.h_lo, a.xb.h_hi);
    const T ex0 = Ex[idx], ey0 = Ey[idx], ez0 = Ez[idx];
    DE<T> d;
    d.zy = (j < ny - 1) ? (Ez[idx + sy] - ez0) : T(0);
    d.yz = (k < nz - 1) ? (Ey[idx + 1] - ey0) : T(0);
    d.xz = (k < nz - 1) ? (Ex[idx + 1] - ex0) : T(0);
    d.zx = (i < nx - 1) ? (Ez[idx + sx] - ez0) : T(0);
    d.yx = (i < nx - 1) ? (Ey[idx + sx] - ey0) : T(0);
    d.xy = (j < ny - 1) ? (Ex[idx + sy] - ex0) : T(0);
    T hx = a.H[0][idx], hy = a.H[1][idx], hz = a.H[2][idx];
    h_cell<T, true>(interior, i, j, k, nx, ny, nz, npml, a.xb, a.dtm, a.dtm_dl, d, a.cph, a.psi_h,
                    a.psi_h, hx, hy, hz);
    a.H_next[0][idx] = hx;
    a.H_next[1][idx] = hy;
    a.H_next[2][idx] = hz;
}

// E^{n+1} of cell (i, j, k) from H_next, E, ψ_E in place, with its sheet
// injections and plane DFTs.  planes is the kernel's __grid_constant__
// parameter.
template <typename T, bool LOSSY>
__device__ __forceinline__ void shell_E_cell(const YeeArgs<T> &a, int i, int j, int k,
                                             const SourceList &src, const PlaneList &planes) {
    const int nx = a.nx, ny = a.ny, nz = a.nz, npml = a.npml;
    const int64_t sx = (int64_t)ny * nz, sy = nz;
    const int64_t idx = (int64_t)i * sx + (int64_t)j * sy + k;
    const T *Hx = a.H_next[0], *Hy = a.H_next[1], *Hz = a.H_next[2];
    const bool interior =
        is_interior(i, j, k, nx, ny, nz, npml, a.xb.e_lo, a.xb.e_hi);
    const T hx0 = Hx[idx], hy0 = Hy[idx], hz0 = Hz[idx];
    DH<T> d;
    d.zy = (j > 0) ? (hz0 - Hz[idx - sy]) : T(0);
    d.yz = (k > 0) ? (hy0 - Hy[idx - 1]) : T(0);
    d.xz = (k > 0) ? (hx0 - Hx[idx - 1]) : T(0);
    d.zx = (i > 0) ? (hz0 - Hz[idx - sx]) : T(0);
    d.yx = (i > 0) ? (hy0 - Hy[idx - sx]) : T(0);
    d.xy = (j > 0) ? (hx0 - Hx[idx - sy]) : T(0);
    const T cex = a.ce[0][idx], cey = a.ce[1][idx], cez = a.ce[2][idx];
    T cax = T(1), cay = T(1), caz = T(1);
    if (LOSSY) {
        cax = a.ca[0][idx];
        cay = a.ca[1][idx];
        caz = a.ca[2][idx];
    }
    T ex = a.E[0][idx], ey = a.E[1][idx], ez = a.E[2][idx];
    if (src.n) ex = apply_sources<T>(src, i, j, k, ex, cex);
    e_cell<T, LOSSY>(interior, i, j, k, nx, ny, nz, npml, a.xb, a.inv_dl, d, a.cpe, a.psi_e, cax, cay,
                     caz, cex, cey, cez, ex, ey, ez);
    a.E_next[0][idx] = ex;
    a.E_next[1][idx] = ey;
    a.E_next[2][idx] = ez;
    if (planes.n && plane_any_hit(planes, i, j, k))
        shell_dft(&planes, i, j, k, nx, ny, nz, (double)ex, (double)ey, (double)ez, (double)hx0,
                  (double)hy0, (double)hz0);
}

template <typename T, bool LOSSY>
__global__ void __launch_bounds__(SHELL_THREADS)
    k_shell_E(YeeArgs<T> a, ShellPlan sp, SourceList src, const __grid_constant__ PlaneList planes) {
    int i, j, k;
    if (!shell_cell(blockIdx.x * SHELL_THREADS + threadIdx.x, sp, i, j, k)) return;
    shell_E_cell<T, LOSSY>(a, i, j, k, src, planes);
}

// The same per-cell E update over the cells of a list of boxes (the shell E
// cells the CPML face kernels do not take: edges, corners and a rim row).
template <typename T, bool LOSSY>
__global__ void __launch_bounds__(SHELL_THREADS)
    k_shell_E_boxes(YeeArgs<T> a, const __grid_constant__ BoxPlan bp, SourceList src,
                    const __grid_constant__ PlaneList planes) {
    int i, j, k;
    if (!box_cell(blockIdx.x * SHELL_THREADS + threadIdx.x, bp, i, j, k)) return;
    shell_E_cell<T, LOSSY>(a, i, j, k, src, planes);
}

// One thread per cell of plane q inside box b: reads E^{n+1}, H^{n+1/2} of the
// cell from E_next / H_next and accumulates the plane's DFT (same arithmetic
// as the E epilogue, so the sums are identical).
template <typename T>
__global__ void __launch_bounds__(SHELL_THREADS)
    k_plane_dft_box(YeeArgs<T> a, ShellBox b, PlaneList planes, int q) {
    const fdtd_plane_dft &p = planes.p[q];
    const int ax = p.axis, u = (ax == 0) ? 1 : 0, w = (ax == 2) ? 1 : 2;
    const int nu = b.hi[u] - b.lo[u], nw = b.hi[w] - b.lo[w];
    const unsigned t = blockIdx.x * SHELL_THREADS + threadIdx.x;
    if (t >= (unsigned)nu * (unsigned)nw) return;
    int c[3];
    c[ax] = p.index;
    c[u] = b.lo[u] + (int)(t / (unsigned)nw);
    c[w] = b.lo[w] + (int)(t % (unsigned)nw);
    const int64_t idx = ((int64_t)c[0] * a.ny + c[1]) * a.nz + c[2];
    double v[6];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        v[m] = (p.comp_mask & (1 << m)) ? (double)a.E_next[m][idx] : 0.0;
        v[m + 3] = (p.comp_mask & (8 << m)) ? (double)a.H_next[m][idx] : 0.0;
    }
    PlaneList one;
    one.p[0] = p;
    one.n = 1;
    plane_dft_cell(one, c[0], c[1], c[2], a.nx, a.ny, a.nz, v);
}

template <typename T>
cudaError_t launch_plane_dft_box(const YeeArgs<T> &a, const ShellBox &b, const PlaneList &pl,
                                 cudaStream_t st) {
    for (int q = 0; q < pl.n; ++q) {
        const int ax = pl.p[q].axis, u = (ax == 0) ? 1 : 0, w = (ax == 2) ? 1 : 2;
        if (pl.p[q].index < b.lo[ax] || pl.p[q].index >= b.hi[ax]) continue;
        const int64_t n = (int64_t)(b.hi[u] - b.lo[u]) * (b.hi[w] - b.lo[w]);
        if (n <= 0) continue;
        k_plane_dft_box<T><<<(unsigned)((n + SHELL_THREADS - 1) / SHELL_THREADS), SHELL_THREADS, 0,
                             st>>>(a, b, pl, q);
        count_launches(1);
    }
    return cudaGetLastError();
}

template cudaError_t launch_plane_dft_box<float>(const YeeArgs<float> &, const ShellBox &,
                                                 const PlaneList &, cudaStream_t);
template cudaError_t launch_plane_dft_box<double>(const YeeArgs<double> &, const ShellBox &,
                                                  const PlaneList &, cudaStream_t);

template <typename T>
cudaError_t launch_shell_H(const YeeArgs<T> &a, const ShellBox &b, cudaStream_t st) {
    const ShellBox o = whole_grid(a.nx, a.ny, a.nz);
    if (!plan_fits(o)) return cudaErrorInvalidConfiguration;
    const ShellPlan sp = make_plan(o, b);
    const unsigned nb = shell_blocks(sp);
    if (nb == 0) return cudaSuccess;
    k_shell_H<T><<<nb, SHELL_THREADS, 0, st>>>(a, sp);
    count_launches(1);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_shell_E_region(const YeeArgs<T> &a, const ShellBox &o, const ShellBox &b,
                                  const SourceList &src, const PlaneList &pl, cudaStream_t st) {
    if (!plan_fits(o)) return cudaErrorInvalidConfiguration;
    const ShellPlan sp = make_plan(o, b);
    const unsigned nb = shell_blocks(sp);
    if (nb == 0) return cudaSuccess;
    if (a.lossy)
        k_shell_E<T, true><<<nb, SHELL_THREADS, 0, st>>>(a, sp, src, pl);
    else
        k_shell_E<T, false><<<nb, SHELL_THREADS, 0, st>>>(a, sp, src, pl);
    count_launches(1);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_shell_E_boxes(const YeeArgs<T> &a, const BoxPlan &bp, const SourceList &src,
                                 const PlaneList &pl, cudaStream_t st) {
    const unsigned nb = plan_blocks(bp);
    if (nb == 0) return cudaSuccess;
    if (a.lossy)
        k_shell_E_boxes<T, true><<<nb, SHELL_THREADS, 0, st>>>(a, bp, src, pl);
    else
        k_shell_E_boxes<T, false><<<nb, SHELL_THREADS, 0, st>>>(a, bp, src, pl);
    count_launches(1);
    return cudaGetLastError();
}

template cudaError_t launch_shell_E_boxes<float>(const YeeArgs<float> &, const BoxPlan &,
                                                 const SourceList &, const PlaneList &,
                                                 cudaStream_t);
template cudaError_t launch_shell_E_boxes<double>(const YeeArgs<double> &, const BoxPlan &,
                                                  const SourceList &, const PlaneList &,
                                                  cudaStream_t);

template <typename T>
cudaError_t launch_shell_E(const YeeArgs<T> &a, const ShellBox &b, const SourceList &src,
                           const PlaneList &pl, cudaStream_t st) {
    return launch_shell_E_region<T>(a, whole_grid(a.nx, a.ny, a.nz), b, src, pl, st);
}

template cudaError_t launch_shell_E_region<float>(const YeeArgs<float> &, const ShellBox &,
                                                  const ShellBox &, const SourceList &,
                                                  const PlaneList &, cudaStream_t);
template cudaError_t launch_shell_E_region<double>(const YeeArgs<double> &, const ShellBox &,
                                                   const ShellBox &, const SourceList &,
                                                   const PlaneList &, cudaStream_t);
template cudaError_t launch_shell_H<float>(const YeeArgs<float> &, const ShellBox &, cudaStream_t);
template cudaError_t launch_shell_H<double>(const YeeArgs<double> &, const ShellBox &,
                                            cudaStream_t);
template cudaError_t launch_shell_E<float>(const YeeArgs<float> &, const ShellBox &,
                                           const SourceList &, const PlaneList &, cudaStream_t);
template cudaError_t launch_shell_E<double>(const YeeArgs<double> &, const ShellBox &,
                                            const SourceList &, const PlaneList &, cudaStream_t);

}  // namespace fdtd
