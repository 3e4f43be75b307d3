// Typed kernel arguments and launcher declarations for the Yee kernels.
#pragma once
#include <cuda_runtime.h>

#include "yee_cell.cuh"

namespace fdtd {

// Everything a Yee kernel needs, by value (device pointers + scalars already
// rounded to T).  E/H are read (and, for the split kernels, written in place);
// E_next/H_next/psi_h_next are the fused kernel's outputs.
template <typename T>
struct YeeArgs {
    int nx, ny, nz, npml, lossy;
    XBounds xb;        // x CPML layers per face and interior x bounds (slabs)
    int ghost_lo, ghost_hi;  // ghost planes at x = 0 / nx-1 (slabs only)
    T dtm, dtm_dl, inv_dl;
    T *E[3];
    T *H[3];
    T *E_next[3];
    T *H_next[3];
    const T *ce[3];
    const T *ca[3];
    Cpml1D<T> cph, cpe;
    T *psi_h[6];
    T *psi_h_next[6];
    T *psi_e[6];
};

// Box [lo, hi) per axis; lo == hi == 0 on every axis means "no box".
struct ShellBox {
    int lo[3], hi[3];
};

template <typename T>
cudaError_t launch_shell_H(const YeeArgs<T> &a, const ShellBox &b, cudaStream_t st);
template <typename T>
cudaError_t launch_shell_E(const YeeArgs<T> &a, const ShellBox &b, const SourceList &src,
                           const PlaneList &pl, cudaStream_t st);
// E^{n+1} of the cells of box o outside box b (b empty: all of o).
template <typename T>
cudaError_t launch_shell_E_region(const YeeArgs<T> &a, const ShellBox &o, const ShellBox &b,
                                  const SourceList &src, const PlaneList &pl, cudaStream_t st);

// Plane-DFT accumulation for the monitored planes' cells inside box b (read
// back from E_next / H_next after the interior update).
template <typename T>
cudaError_t launch_plane_dft_box(const YeeArgs<T> &a, const ShellBox &b, const PlaneList &pl,
                                 cudaStream_t st);

struct SideStream;

// Shell E of the fused step through the CPML face kernels (yee_face.cu): the
// six face slabs as TMA plane marches on st, the remaining shell cells by the
// per-cell kernel on the side stream, joined back to st; no plane DFTs (the
// caller accumulates the monitored planes afterwards); cudaErrorNotSupported,
// with nothing launched, when the tensor maps cannot be built.  face_path_ok:
// the grid qualifies (whole grid, npml a multiple of 16 bytes of elements,
// aligned stripes).
template <typename T>
bool face_path_ok(const YeeArgs<T> &a);
template <typename T>
cudaError_t launch_shell_E_faces(const YeeArgs<T> &a, const SourceList &src, cudaStream_t st,
                                 SideStream *side);
int read_face_error(int reset);
unsigned interior_wait_polls();

template <typename T>
cudaError_t launch_update_H(const YeeArgs<T> &a, cudaStream_t st);
template <typename T>
cudaError_t launch_update_E(const YeeArgs<T> &a, const SourceList &src, const PlaneList &pl,
                            cudaStream_t st);
template <typename T>
cudaError_t launch_add_source(int nx, int ny, int nz, const fdtd_source &s, T *Ex,
                              const T *ce_x, cudaStream_t st);
// Fused step: shell H, interior single-pass kernel, shell E.  Reads E/H/psi,
// writes E_next/H_next (psi in place).  Falls back to the shell kernels over
// the whole grid when the interior kernel's TMA alignment does not hold.
template <typename T>
cudaError_t launch_step_fused(const YeeArgs<T> &a, const SourceList &src, const PlaneList &pl,
                              cudaStream_t st);

}  // namespace fdtd
