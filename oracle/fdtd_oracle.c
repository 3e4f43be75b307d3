/*
 * CPU oracle for the FDTD Yee/CPML time step — TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the arithmetic of the reference OpenCL
 * kernels so that the CUDA path can be checked against it on identical inputs:
 *
 *   H update, interior cells  : opencl_fdtd_solver/kernels/yee_update.cl:11-40
 *   H update, CPML cells      : opencl_fdtd_solver/kernels/yee_update.cl:42-118
 *   E update, interior cells  : opencl_fdtd_solver/kernels/yee_update.cl:120-155
 *   E update, CPML cells      : opencl_fdtd_solver/kernels/yee_update.cl:157-238
 *   Jx sheet source           : opencl_fdtd_solver/kernels/sources.cl:26-49
 *   Ex soft source (legacy)   : opencl_fdtd_solver/kernels/sources.cl:7-21
 *   launch split and folding  : opencl_fdtd_solver/engine.py:540-722
 *
 * A cell is "interior" when npml > 0 and all three indices lie in
 * [npml, N - npml); interior cells use the folded dt/(mu0*dl) and ce*(1/dl)
 * forms, every other cell uses the kappa/psi form with boundary-guarded
 * differences, exactly as the reference's two launches per half step do.
 *
 * Build with -ffp-contract=off: every product and sum is rounded separately,
 * so results are deterministic and independent of the thread count.
 * Nothing in the product links this file; only tests/, __graft_entry__.smoke()
 * and the CPU-baseline leg of bench.py load it, as the checker.
 */
#include <stddef.h>
#include <stdint.h>

#define OG_INTERIOR(i, j, k)                                                  \
    (npml > 0 && (i) >= npml && (i) < nx - npml && (j) >= npml &&             \
     (j) < ny - npml && (k) >= npml && (k) < nz - npml)

/* Face-stripe index of a PML cell along one axis: low face layers 0..npml-1,
 * high face layers npml..2npml-1 (yee_update.cl:91,99,107). */
#define OG_LAYER(x, n) (((x) < npml) ? (x) : (npml + (x) - ((n) - npml)))

#define OG_DEFINE(T, SUF)                                                      \
void og_update_H_##SUF(                                                        \
    int nx, int ny, int nz, int npml, T dtm, T dtm_dl,                         \
    const T *Ex, const T *Ey, const T *Ez, T *Hx, T *Hy, T *Hz,                \
    const T *bx, const T *cx, const T *ikx,                                    \
    const T *by, const T *cy, const T *iky,                                    \
    const T *bz, const T *cz, const T *ikz,                                    \
    T *psi_Hx_y, T *psi_Hx_z, T *psi_Hy_x, T *psi_Hy_z,                        \
    T *psi_Hz_x, T *psi_Hz_y)                                                  \
{                                                                              \
    const int64_t sx = (int64_t)ny * nz, sy = nz;                              \
    _Pragma("omp parallel for collapse(2) schedule(static)")                   \
    for (int i = 0; i < nx; ++i)                                               \
    for (int j = 0; j < ny; ++j) {                                             \
        for (int k = 0; k < nz; ++k) {                                         \
            const int64_t idx = i * sx + j * sy + k;                           \
            if (OG_INTERIOR(i, j, k)) {                                        \
                T dEz_dy = Ez[idx + sy] - Ez[idx];                             \
                T dEy_dz = Ey[idx + 1] - Ey[idx];                              \
                T dEx_dz = Ex[idx + 1] - Ex[idx];                              \
                T dEz_dx = Ez[idx + sx] - Ez[idx];                             \
                T dEy_dx = Ey[idx + sx] - Ey[idx];                             \
                T dEx_dy = Ex[idx + sy] - Ex[idx];                             \
                Hx[idx] = Hx[idx] - dtm_dl * (dEz_dy - dEy_dz);                \
                Hy[idx] = Hy[idx] - dtm_dl * (dEx_dz - dEz_dx);                \
                Hz[idx] = Hz[idx] - dtm_dl * (dEy_dx - dEx_dy);                \
                continue;                                                      \
            }                                                                  \
            T dEz_dy = (j < ny - 1) ? (Ez[idx + sy] - Ez[idx]) : (T)0;         \
            T dEy_dz = (k < nz - 1) ? (Ey[idx + 1] - Ey[idx]) : (T)0;          \
            T dEx_dz = (k < nz - 1) ? (Ex[idx + 1] - Ex[idx]) : (T)0;          \
            T dEz_dx = (i < nx - 1) ? (Ez[idx + sx] - Ez[idx]) : (T)0;         \
            T dEy_dx = (i < nx - 1) ? (Ey[idx + sx] - Ey[idx]) : (T)0;         \
            T dEx_dy = (j < ny - 1) ? (Ex[idx + sy] - Ex[idx]) : (T)0;         \
            T p_Hx_y = 0, p_Hx_z = 0, p_Hy_x = 0, p_Hy_z = 0;                  \
            T p_Hz_x = 0, p_Hz_y = 0;                                          \
            if (npml > 0 && (i < npml || i >= nx - npml)) {                    \
                int64_t s = (int64_t)OG_LAYER(i, nx) * sx + j * sy + k;        \
                p_Hy_x = bx[i] * psi_Hy_x[s] + cx[i] * dEz_dx;                 \
                p_Hz_x = bx[i] * psi_Hz_x[s] + cx[i] * dEy_dx;                 \
                psi_Hy_x[s] = p_Hy_x;                                          \
                psi_Hz_x[s] = p_Hz_x;                                          \
            }                                                                  \
            if (npml > 0 && (j < npml || j >= ny - npml)) {                    \
                int64_t s = (int64_t)i * (2 * npml) * nz +                     \
                            (int64_t)OG_LAYER(j, ny) * nz + k;                 \
                p_Hx_y = by[j] * psi_Hx_y[s] + cy[j] * dEz_dy;                 \
                p_Hz_y = by[j] * psi_Hz_y[s] + cy[j] * dEx_dy;                 \
                psi_Hx_y[s] = p_Hx_y;                                          \
                psi_Hz_y[s] = p_Hz_y;                                          \
            }                                                                  \
            if (npml > 0 && (k < npml || k >= nz - npml)) {                    \
                int64_t s = ((int64_t)i * ny + j) * (2 * npml) +               \
                            OG_LAYER(k, nz);                                   \
                p_Hx_z = bz[k] * psi_Hx_z[s] + cz[k] * dEy_dz;                 \
                p_Hy_z = bz[k] * psi_Hy_z[s] + cz[k] * dEx_dz;                 \
                psi_Hx_z[s] = p_Hx_z;                                          \
                psi_Hy_z[s] = p_Hy_z;                                          \
            }                                                                  \
            Hx[idx] = Hx[idx] -                                                \
                dtm * (dEz_dy * iky[j] + p_Hx_y - dEy_dz * ikz[k] - p_Hx_z);   \
            Hy[idx] = Hy[idx] -                                                \
                dtm * (dEx_dz * ikz[k] + p_Hy_z - dEz_dx * ikx[i] - p_Hy_x);   \
            Hz[idx] = Hz[idx] -                                                \
                dtm * (dEy_dx * ikx[i] + p_Hz_x - dEx_dy * iky[j] - p_Hz_y);   \
        }                                                                      \
    }                                                                          \
}                                                                              \
                                                                               \
void og_update_E_##SUF(                                                        \
    int nx, int ny, int nz, int npml, T inv_dl,                                \
    const T *ca_x, const T *ca_y, const T *ca_z,                               \
    const T *ce_x, const T *ce_y, const T *ce_z,                               \
    const T *Hx, const T *Hy, const T *Hz, T *Ex, T *Ey, T *Ez,                \
    const T *bx, const T *cx, const T *ikx,                                    \
    const T *by, const T *cy, const T *iky,                                    \
    const T *bz, const T *cz, const T *ikz,                                    \
    T *psi_Ex_y, T *psi_Ex_z, T *psi_Ey_x, T *psi_Ey_z,                        \
    T *psi_Ez_x, T *psi_Ez_y)                                                  \
{                                                                              \
    const int64_t sx = (int64_t)ny * nz, sy = nz;                              \
    _Pragma("omp parallel for collapse(2) schedule(static)")                   \
    for (int i = 0; i < nx; ++i)                                               \
    for (int j = 0; j < ny; ++j) {                                             \
        for (int k = 0; k < nz; ++k) {                                         \
            const int64_t idx = i * sx + j * sy + k;                           \
            if (OG_INTERIOR(i, j, k)) {                                        \
                T dHz_dy = Hz[idx] - Hz[idx - sy];                             \
                T dHy_dz = Hy[idx] - Hy[idx - 1];                              \
                T dHx_dz = Hx[idx] - Hx[idx - 1];                              \
                T dHz_dx = Hz[idx] - Hz[idx - sx];                             \
                T dHy_dx = Hy[idx] - Hy[idx - sx];                             \
                T dHx_dy = Hx[idx] - Hx[idx - sy];                             \
                Ex[idx] = ca_x[idx] * Ex[idx] +                                \
                          ce_x[idx] * inv_dl * (dHz_dy - dHy_dz);              \
                Ey[idx] = ca_y[idx] * Ey[idx] +                                \
                          ce_y[idx] * inv_dl * (dHx_dz - dHz_dx);              \
                Ez[idx] = ca_z[idx] * Ez[idx] +                                \
                          ce_z[idx] * inv_dl * (dHy_dx - dHx_dy);              \
                continue;                                                      \
            }                                                                  \
            T dHz_dy = (j > 0) ? (Hz[idx] - Hz[idx - sy]) : (T)0;              \
            T dHy_dz = (k > 0) ? (Hy[idx] - Hy[idx - 1]) : (T)0;               \
            T dHx_dz = (k > 0) ? (Hx[idx] - Hx[idx - 1]) : (T)0;               \
            T dHz_dx = (i > 0) ? (Hz[idx] - Hz[idx - sx]) : (T)0;              \
            T dHy_dx = (i > 0) ? (Hy[idx] - Hy[idx - sx]) : (T)0;              \
            T dHx_dy = (j > 0) ? (Hx[idx] - Hx[idx - sy]) : (T)0;              \
            T p_Ex_y = 0, p_Ex_z = 0, p_Ey_x = 0, p_Ey_z = 0;                  \
            T p_Ez_x = 0, p_Ez_y = 0;                                          \
            if (npml > 0 && (i < npml || i >= nx - npml)) {                    \
                int64_t s = (int64_t)OG_LAYER(i, nx) * sx + j * sy + k;        \
                p_Ey_x = bx[i] * psi_Ey_x[s] + cx[i] * dHz_dx;                 \
                p_Ez_x = bx[i] * psi_Ez_x[s] + cx[i] * dHy_dx;                 \
                psi_Ey_x[s] = p_Ey_x;                                          \
                psi_Ez_x[s] = p_Ez_x;                                          \
            }                                                                  \
            if (npml > 0 && (j < npml || j >= ny - npml)) {                    \
                int64_t s = (int64_t)i * (2 * npml) * nz +                     \
                            (int64_t)OG_LAYER(j, ny) * nz + k;                 \
                p_Ex_y = by[j] * psi_Ex_y[s] + cy[j] * dHz_dy;                 \
                p_Ez_y = by[j] * psi_Ez_y[s] + cy[j] * dHx_dy;                 \
                psi_Ex_y[s] = p_Ex_y;                                          \
                psi_Ez_y[s] = p_Ez_y;                                          \
            }                                                                  \
            if (npml > 0 && (k < npml || k >= nz - npml)) {                    \
                int64_t s = ((int64_t)i * ny + j) * (2 * npml) +               \
                            OG_LAYER(k, nz);                                   \
                p_Ex_z = bz[k] * psi_Ex_z[s] + cz[k] * dHy_dz;                 \
                p_Ey_z = bz[k] * psi_Ey_z[s] + cz[k] * dHx_dz;                 \
                psi_Ex_z[s] = p_Ex_z;                                          \
                psi_Ey_z[s] = p_Ey_z;                                          \
            }                                                                  \
            Ex[idx] = ca_x[idx] * Ex[idx] + ce_x[idx] *                        \
                (dHz_dy * iky[j] + p_Ex_y - dHy_dz * ikz[k] - p_Ex_z);         \
            Ey[idx] = ca_y[idx] * Ey[idx] + ce_y[idx] *                        \
                (dHx_dz * ikz[k] + p_Ey_z - dHz_dx * ikx[i] - p_Ey_x);         \
            Ez[idx] = ca_z[idx] * Ez[idx] + ce_z[idx] *                        \
                (dHy_dx * ikx[i] + p_Ez_x - dHx_dy * iky[j] - p_Ez_y);         \
        }                                                                      \
    }                                                                          \
}                                                                              \
                                                                               \
void og_source_Jx_##SUF(                                                       \
    int nx, int ny, int nz, int z_src, T jx, int i0, int i1, int j0, int j1,   \
    int rim_taper, T rim_edge, const T *ce_x, T *Ex)                           \
{                                                                              \
    if (z_src < 0 || z_src >= nz) return;                                      \
    for (int i = (i0 > 0 ? i0 : 0); i < i1 && i < nx; ++i)                     \
    for (int j = (j0 > 0 ? j0 : 0); j < j1 && j < ny; ++j) {                   \
        T w = (T)1;                                                            \
        if (rim_taper) {                                                       \
            if (i == i0 || i == i1 - 1) w = w * rim_edge;                      \
            if (j == j0 || j == j1 - 1) w = w * rim_edge;                      \
        }                                                                      \
        int64_t idx = ((int64_t)i * ny + j) * nz + z_src;                      \
        Ex[idx] = Ex[idx] + -ce_x[idx] * jx * w;                               \
    }                                                                          \
}                                                                              \
                                                                               \
void og_source_Ex_##SUF(                                                       \
    int nx, int ny, int nz, int z_src, T amp, int i0, int i1, int j0, int j1,  \
    T *Ex)                                                                     \
{                                                                              \
    if (z_src < 0 || z_src >= nz) return;                                      \
    for (int i = (i0 > 0 ? i0 : 0); i < i1 && i < nx; ++i)                     \
    for (int j = (j0 > 0 ? j0 : 0); j < j1 && j < ny; ++j) {                   \
        int64_t idx = ((int64_t)i * ny + j) * nz + z_src;                      \
        Ex[idx] = Ex[idx] + amp;                                               \
    }                                                                          \
}

OG_DEFINE(float, f32)
OG_DEFINE(double, f64)

/* Thread count actually used by the OpenMP runtime (reported with baselines). */
#ifdef _OPENMP
#include <omp.h>
int og_num_threads(void) { return omp_get_max_threads(); }
void og_set_num_threads(int n) { if (n > 0) omp_set_num_threads(n); }
#else
int og_num_threads(void) { return 1; }
void og_set_num_threads(int n) { (void)n; }
#endif
