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

template <typename T>
cudaError_t launch_update_H(const YeeArgs<T> &a, cudaStream_t st);
template <typename T>
cudaError_t launch_update_E(const YeeArgs<T> &a, const SourceList &src, const PlaneList &pl,
                            cudaStream_t st);
template <typename T>
cudaError_t launch_add_source(int nx, int ny, int nz, const fdtd_source &s, T *Ex,
                              const T *ce_x, cudaStream_t st);
// Fused single-pass step; returns cudaErrorNotSupported when the shape or the
// alignment does not admit the fused schedule (the caller then runs H and E).
template <typename T>
cudaError_t launch_step_fused(const YeeArgs<T> &a, const SourceList &src, const PlaneList &pl,
                              cudaStream_t st);

}  // namespace fdtd
