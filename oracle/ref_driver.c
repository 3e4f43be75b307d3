/*
 * Host driver for the reference's own Yee/source kernels compiled as C
 * (TEST INFRASTRUCTURE ONLY; built into oracle/_ref/, never shipped).
 *
 * The kernel files are #included from the reference tree at build time (the
 * include path is given by oracle/Makefile); nothing of them is copied here.
 * The driver enqueues them the way OpenCLFDTD does (engine.py:540-722): when
 * npml > 0 the interior kernel runs over [npml, N-npml)^3 and then the PML
 * kernel over the whole grid (its interior work-items return at once); when
 * npml == 0 only the guarded PML kernel runs.  Work-items run as OpenMP
 * iterations; the padding work-items of the reference's NDRange return
 * immediately in the kernels, so they are not visited.
 *
 * Compiled twice: -DUSE_FP64=0 -DREF_SUF=f32 and -DUSE_FP64=1 -DREF_SUF=f64.
 */
#include "ref_shim.h"
#include "precision.cl"
#include "yee_update.cl"
#include "sources.cl"

#define REF_CAT2(a, b) a##_##b
#define REF_CAT(a, b) REF_CAT2(a, b)
#define REF(name) REF_CAT(ref_##name, REF_SUF)

#define REF_FOR3(NI, NJ, NK, BODY)                                            \
    _Pragma("omp parallel for collapse(2) schedule(static)")                  \
    for (int gi = 0; gi < (NI); ++gi)                                         \
        for (int gj = 0; gj < (NJ); ++gj)                                     \
            for (int gk = 0; gk < (NK); ++gk) {                               \
                ref_gid[0] = (size_t)gk;                                      \
                ref_gid[1] = (size_t)gj;                                      \
                ref_gid[2] = (size_t)gi;                                      \
                BODY;                                                         \
            }

void REF(update_H)(int nx, int ny, int nz, int npml, real dtm, real dtm_dl,
                   const real *Ex, const real *Ey, const real *Ez,
                   real *Hx, real *Hy, real *Hz,
                   const real *bx, const real *cx, const real *ikx,
                   const real *by, const real *cy, const real *iky,
                   const real *bz, const real *cz, const real *ikz,
                   real *psi_Hx_y, real *psi_Hx_z, real *psi_Hy_x,
                   real *psi_Hy_z, real *psi_Hz_x, real *psi_Hz_y)
{
    int ni = nx - 2 * npml, nj = ny - 2 * npml, nk = nz - 2 * npml;
    if (npml > 0 && ni > 0 && nj > 0 && nk > 0) {
        REF_FOR3(ni, nj, nk,
                 update_H_interior(nx, ny, nz, npml, dtm_dl, Ex, Ey, Ez, Hx, Hy, Hz));
    }
    REF_FOR3(nx, ny, nz,
             update_H_pml(nx, ny, nz, npml, dtm, Ex, Ey, Ez, Hx, Hy, Hz,
                          bx, cx, ikx, by, cy, iky, bz, cz, ikz,
                          psi_Hx_y, psi_Hx_z, psi_Hy_x, psi_Hy_z, psi_Hz_x, psi_Hz_y));
}

void REF(update_E)(int nx, int ny, int nz, int npml, real inv_dl,
                   const real *ca_x, const real *ca_y, const real *ca_z,
                   const real *ce_x, const real *ce_y, const real *ce_z,
                   const real *Hx, const real *Hy, const real *Hz,
                   real *Ex, real *Ey, real *Ez,
                   const real *bx, const real *cx, const real *ikx,
                   const real *by, const real *cy, const real *iky,
                   const real *bz, const real *cz, const real *ikz,
                   real *psi_Ex_y, real *psi_Ex_z, real *psi_Ey_x,
                   real *psi_Ey_z, real *psi_Ez_x, real *psi_Ez_y)
{
    int ni = nx - 2 * npml, nj = ny - 2 * npml, nk = nz - 2 * npml;
    if (npml > 0 && ni > 0 && nj > 0 && nk > 0) {
        REF_FOR3(ni, nj, nk,
                 update_E_interior(nx, ny, nz, npml, inv_dl, ca_x, ca_y, ca_z,
                                   ce_x, ce_y, ce_z, Hx, Hy, Hz, Ex, Ey, Ez));
    }
    REF_FOR3(nx, ny, nz,
             update_E_pml(nx, ny, nz, npml, ca_x, ca_y, ca_z, ce_x, ce_y, ce_z,
                          Hx, Hy, Hz, Ex, Ey, Ez,
                          bx, cx, ikx, by, cy, iky, bz, cz, ikz,
                          psi_Ex_y, psi_Ex_z, psi_Ey_x, psi_Ey_z, psi_Ez_x, psi_Ez_y));
}

void REF(source_Jx)(int nx, int ny, int nz, int z_src, real jx, int i0, int i1,
                    int j0, int j1, int rim_taper, real rim_edge,
                    const real *ce_x, real *Ex)
{
    /* NDRange (Ny, Nx): id0 = j, id1 = i (engine.py:521-538). */
    for (int gi = 0; gi < nx; ++gi)
        for (int gj = 0; gj < ny; ++gj) {
            ref_gid[0] = (size_t)gj;
            ref_gid[1] = (size_t)gi;
            add_source_Jx(nx, ny, nz, z_src, jx, i0, i1, j0, j1, rim_taper,
                          rim_edge, ce_x, Ex);
        }
}

void REF(source_Ex)(int nx, int ny, int nz, int z_src, real amp, int i0, int i1,
                    int j0, int j1, real *Ex)
{
    for (int gi = 0; gi < nx; ++gi)
        for (int gj = 0; gj < ny; ++gj) {
            ref_gid[0] = (size_t)gj;
            ref_gid[1] = (size_t)gi;
            add_source_Ex(nx, ny, nz, z_src, amp, i0, i1, j0, j1, Ex);
        }
}
