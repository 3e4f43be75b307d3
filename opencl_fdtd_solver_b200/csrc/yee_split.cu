// Split half-step kernels: H update, E update (+ sheet injections and plane
// DFTs in its epilogue) and an immediate sheet injection.  One thread per cell,
// (k, j) thread blocks so that each warp reads 32 consecutive k (128-byte rows
// in FP32).  These run when a source callback needs H^{n+1/2} materialised
// before E is updated, and for the immediate-injection path; the normal step
// is the fused kernel in yee_fused.cu.
//
// Compiled with --fmad=false (see build.py) so each cell rounds exactly as the
// reference kernels with every operation rounded separately.
#include <cuda_runtime.h>

#include "launch_count.cuh"
#include "yee_cell.cuh"
#include "yee_launch.cuh"

namespace fdtd {

constexpr int SPLIT_TK = 32;
constexpr int SPLIT_TJ = 8;

template <typename T>
__global__ void __launch_bounds__(SPLIT_TK *SPLIT_TJ)
    k_update_H(YeeArgs<T> a) {
    const int k = blockIdx.x * SPLIT_TK + threadIdx.x;
    const int j = blockIdx.y * SPLIT_TJ + threadIdx.y;
    const int i = blockIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz, npml = a.npml;
    if (k >= nz || j >= ny) return;
    const int64_t sx = (int64_t)ny * nz, sy = nz;
    const int64_t idx = (int64_t)i * sx + (int64_t)j * sy + k;
    const T *Ex = a.E[0], *Ey = a.E[1], *Ez = a.E[2];
    const bool interior =
        is_interior(i, j, k, nx, ny, nz, npml, a.xb.h_lo, a.xb.h_hi);
    DE<T> d;
    const T ex0 = Ex[idx], ey0 = Ey[idx], ez0 = Ez[idx];
    if (interior) {
        d.zy = Ez[idx + sy] - ez0;
        d.yz = Ey[idx + 1] - ey0;
        d.xz = Ex[idx + 1] - ex0;
        d.zx = Ez[idx + sx] - ez0;
        d.yx = Ey[idx + sx] - ey0;
        d.xy = Ex[idx + sy] - ex0;
    } else {
        d.zy = (j < ny - 1) ? (Ez[idx + sy] - ez0) : T(0);
        d.yz = (k < nz - 1) ? (Ey[idx + 1] - ey0) : T(0);
        d.xz = (k < nz - 1) ? (Ex[idx + 1] - ex0) : T(0);
        d.zx = (i < nx - 1) ? (Ez[idx + sx] - ez0) : T(0);
        d.yx = (i < nx - 1) ? (Ey[idx + sx] - ey0) : T(0);
        d.xy = (j < ny - 1) ? (Ex[idx + sy] - ex0) : T(0);
    }
    T hx = a.H[0][idx], hy = a.H[1][idx], hz = a.H[2][idx];
    h_cell<T>(interior, i, j, k, nx, ny, nz, npml, a.xb, a.dtm, a.dtm_dl, d, a.cph, a.psi_h,
              a.psi_h, hx, hy, hz);
    a.H[0][idx] = hx;
    a.H[1][idx] = hy;
    a.H[2][idx] = hz;
}

template <typename T, bool LOSSY>
__global__ void __launch_bounds__(SPLIT_TK *SPLIT_TJ)
    k_update_E(YeeArgs<T> a, SourceList src, PlaneList planes) {
    const int k = blockIdx.x * SPLIT_TK + threadIdx.x;
    const int j = blockIdx.y * SPLIT_TJ + threadIdx.y;
    const int i = blockIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz, npml = a.npml;
    if (k >= nz || j >= ny) return;
    const int64_t sx = (int64_t)ny * nz, sy = nz;
    const int64_t idx = (int64_t)i * sx + (int64_t)j * sy + k;
    const T *Hx = a.H[0], *Hy = a.H[1], *Hz = a.H[2];
    const bool interior =
        is_interior(i, j, k, nx, ny, nz, npml, a.xb.e_lo, a.xb.e_hi);
    const T hx0 = Hx[idx], hy0 = Hy[idx], hz0 = Hz[idx];
    DH<T> d;
    if (interior) {
        d.zy = hz0 - Hz[idx - sy];
        d.yz = hy0 - Hy[idx - 1];
        d.xz = hx0 - Hx[idx - 1];
        d.zx = hz0 - Hz[idx - sx];
        d.yx = hy0 - Hy[idx - sx];
        d.xy = hx0 - Hx[idx - sy];
    } else {
        d.zy = (j > 0) ? (hz0 - Hz[idx - sy]) : T(0);
        d.yz = (k > 0) ? (hy0 - Hy[idx - 1]) : T(0);
        d.xz = (k > 0) ? (hx0 - Hx[idx - 1]) : T(0);
        d.zx = (i > 0) ? (hz0 - Hz[idx - sx]) : T(0);
        d.yx = (i > 0) ? (hy0 - Hy[idx - sx]) : T(0);
        d.xy = (j > 0) ? (hx0 - Hx[idx - sy]) : T(0);
    }
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
    a.E[0][idx] = ex;
    a.E[1][idx] = ey;
    a.E[2][idx] = ez;
    if (planes.n && plane_any_hit(planes, i, j, k)) {
        const double v[6] = {(double)ex, (double)ey, (double)ez,
                             (double)hx0, (double)hy0, (double)hz0};
        plane_dft_cell(planes, i, j, k, nx, ny, nz, v);
    }
}

template <typename T>
__global__ void k_add_source(int nx, int ny, int nz, fdtd_source s, T *Ex, const T *ce_x) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= ny || i >= nx) return;
    if (i < s.i0 || i >= s.i1 || j < s.j0 || j >= s.j1) return;
    const int64_t idx = ((int64_t)i * ny + j) * nz + s.z;
    SourceList one;
    one.s[0] = s;
    one.n = 1;
    Ex[idx] = apply_sources<T>(one, i, j, s.z, Ex[idx], ce_x[idx]);
}

template <typename T>
cudaError_t launch_update_H(const YeeArgs<T> &a, cudaStream_t st) {
    dim3 blk(SPLIT_TK, SPLIT_TJ, 1);
    dim3 grd((a.nz + SPLIT_TK - 1) / SPLIT_TK, (a.ny + SPLIT_TJ - 1) / SPLIT_TJ, a.nx);
    k_update_H<T><<<grd, blk, 0, st>>>(a);
    count_launches(1);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_update_E(const YeeArgs<T> &a, const SourceList &src, const PlaneList &pl,
                            cudaStream_t st) {
    dim3 blk(SPLIT_TK, SPLIT_TJ, 1);
    dim3 grd((a.nz + SPLIT_TK - 1) / SPLIT_TK, (a.ny + SPLIT_TJ - 1) / SPLIT_TJ, a.nx);
    if (a.lossy)
        k_update_E<T, true><<<grd, blk, 0, st>>>(a, src, pl);
    else
        k_update_E<T, false><<<grd, blk, 0, st>>>(a, src, pl);
    count_launches(1);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_add_source(int nx, int ny, int nz, const fdtd_source &s, T *Ex,
                              const T *ce_x, cudaStream_t st) {
    dim3 blk(128, 1, 1);
    dim3 grd((ny + 127) / 128, nx, 1);
    k_add_source<T><<<grd, blk, 0, st>>>(nx, ny, nz, s, Ex, ce_x);
    count_launches(1);
    return cudaGetLastError();
}

template cudaError_t launch_update_H<float>(const YeeArgs<float> &, cudaStream_t);
template cudaError_t launch_update_H<double>(const YeeArgs<double> &, cudaStream_t);
template cudaError_t launch_update_E<float>(const YeeArgs<float> &, const SourceList &,
                                            const PlaneList &, cudaStream_t);
template cudaError_t launch_update_E<double>(const YeeArgs<double> &, const SourceList &,
                                             const PlaneList &, cudaStream_t);
template cudaError_t launch_add_source<float>(int, int, int, const fdtd_source &, float *,
                                              const float *, cudaStream_t);
template cudaError_t launch_add_source<double>(int, int, int, const fdtd_source &, double *,
                                               const double *, cudaStream_t);

}  // namespace fdtd
