// Adjoint-sweep kernel arguments and launchers (adjoint.cu).
#pragma once
#include <cuda_runtime.h>

#include "yee_cell.cuh"

namespace fdtd {

// Adjoint state and the forward coefficients it needs, by value.
template <typename T>
struct AdjArgs {
    int nx, ny, nz, npml;
    T dtm;
    T *E[3];
    T *H[3];
    const T *ce[3];
    const T *pe[6];
    T *pe_next[6];
    const T *ph[6];
    T *ph_next[6];
    Cpml1D<T> cph, cpe;
};

struct AdjSeed {
    int active;
    int axis, index, a0, a1, b0, b1, comp_mask, nfreq;
    const double *seed;
    const double *phase;
};

template <typename T>
struct AdjGrad {
    int active;
    int lo[3], hi[3];
    const T *e_next, *e_prev;
    double *g;
};

// Transposed E update then transposed H update (one reverse step), then sd.
template <typename T>
cudaError_t launch_adjoint_step(const AdjArgs<T> &a, const AdjGrad<T> &gb, const AdjSeed &sd,
                                cudaStream_t st);
template <typename T>
cudaError_t launch_adjoint_seed(int nx, int ny, int nz, T *const E[3], const AdjSeed &sd,
                                cudaStream_t st);
template <typename T>
cudaError_t launch_capture(int ny, int nz, const T *const E[3], const int lo[3], const int hi[3],
                           T *out, cudaStream_t st);

}  // namespace fdtd
