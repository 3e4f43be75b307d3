// Adjoint-sweep kernel arguments and launchers (adjoint.cu).
#pragma once
#include <cuda_runtime.h>

#include "yee_launch.cuh"

namespace fdtd {

// Adjoint state and the forward coefficients it needs, by value.
template <typename T>
struct AdjArgs {
    int nx, ny, nz, npml;
    T dtm;
    T ik_int;  // 1/(κ·dl) of the CPML-free interior (κ = 1), rounded to T
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

// Where a reverse step writes: H̄ and Ē (== AdjArgs::H / E for in place).
template <typename T>
struct AdjOut {
    T *E[3];
    T *H[3];
};

// Transposed E update then transposed H update (one reverse step), then sd.
template <typename T>
cudaError_t launch_adjoint_step(const AdjArgs<T> &a, const AdjGrad<T> &gb, const AdjSeed &sd,
                                cudaStream_t st);
// The same step with H̄ written to out.H and Ē to out.E (grid-wide kernels).
template <typename T>
cudaError_t launch_adjoint_grid(const AdjArgs<T> &a, const AdjGrad<T> &gb, const AdjSeed &sd,
                                const AdjOut<T> &out, cudaStream_t st);
// The half steps on the cells of box o outside box b only (no seed).
template <typename T>
cudaError_t launch_adjoint_shell_H(const AdjArgs<T> &a, const AdjGrad<T> &gb, const AdjOut<T> &out,
                                   const ShellBox &o, const ShellBox &b, cudaStream_t st);
template <typename T>
cudaError_t launch_adjoint_shell_E(const AdjArgs<T> &a, const AdjOut<T> &out, const ShellBox &o,
                                   const ShellBox &b, cudaStream_t st);
// The fused reverse step: interior march (adjoint_fused.cu) beside the shell
// kernels; reads a.E / a.H, writes out.E / out.H, then adds the seed.
template <typename T>
cudaError_t launch_adjoint_step_fused(const AdjArgs<T> &a, const AdjGrad<T> &gb,
                                      const AdjSeed &sd, const AdjOut<T> &out, cudaStream_t st);
int read_adjoint_error(int reset);
template <typename T>
cudaError_t launch_adjoint_seed(int nx, int ny, int nz, T *const E[3], const AdjSeed &sd,
                                cudaStream_t st);
template <typename T>
cudaError_t launch_capture(int ny, int nz, const T *const E[3], const int lo[3], const int hi[3],
                           T *out, cudaStream_t st);

}  // namespace fdtd
