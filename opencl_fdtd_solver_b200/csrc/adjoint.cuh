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

// Objective seed for E cell (i, j, k): Ē_c += Σ_f Re(seed)·Re(phase) + Im(seed)·Im(phase).
template <typename T>
__device__ __forceinline__ void add_seed(const AdjSeed &sd, int i, int j, int k, T &ex, T &ey,
                                         T &ez) {
    const int w = sd.axis == 0 ? i : (sd.axis == 1 ? j : k);
    if (w != sd.index) return;
    const int pa = sd.axis == 0 ? j : i;
    const int pb = sd.axis == 2 ? j : k;
    if (pa < sd.a0 || pa >= sd.a1 || pb < sd.b0 || pb >= sd.b1) return;
    const int64_t np = (int64_t)(sd.a1 - sd.a0) * (sd.b1 - sd.b0);
    const int64_t loc = (int64_t)(pa - sd.a0) * (sd.b1 - sd.b0) + (pb - sd.b0);
    int slot = 0;
    for (int c = 0; c < 3; ++c) {
        if (!(sd.comp_mask & (1 << c))) continue;
        double acc = 0.0;
        for (int f = 0; f < sd.nfreq; ++f) {
            const double *s = sd.seed + 2 * (((int64_t)slot * sd.nfreq + f) * np + loc);
            acc = acc + (s[0] * sd.phase[2 * f] + s[1] * sd.phase[2 * f + 1]);
        }
        if (c == 0) ex = ex + (T)acc;
        if (c == 1) ey = ey + (T)acc;
        if (c == 2) ez = ez + (T)acc;
        ++slot;
    }
}

// G_c += Ē_c·(E_c^{n+1} − E_c^n) for a cell of the gradient box.
template <typename T>
__device__ __forceinline__ void adj_grad_cell(const AdjGrad<T> &gb, int i, int j, int k, T ex,
                                              T ey, T ez) {
    if (i < gb.lo[0] || i >= gb.hi[0] || j < gb.lo[1] || j >= gb.hi[1] || k < gb.lo[2] ||
        k >= gb.hi[2])
        return;
    const int by = gb.hi[1] - gb.lo[1], bz = gb.hi[2] - gb.lo[2];
    const int64_t nb = (int64_t)(gb.hi[0] - gb.lo[0]) * by * bz;
    const int64_t loc = ((int64_t)(i - gb.lo[0]) * by + (j - gb.lo[1])) * bz + (k - gb.lo[2]);
    const T ev[3] = {ex, ey, ez};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int64_t q = c * nb + loc;
        const double de = (double)gb.e_next[q] - (double)gb.e_prev[q];
        gb.g[q] = gb.g[q] + (double)ev[c] * de;
    }
}

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
// The half steps on the cells of box o outside box b only; the H̄ launch also
// accumulates the gradient of the cells of box gx (empty: none), the Ē launch
// adds the seed sd of its cells.
template <typename T>
cudaError_t launch_adjoint_shell_H(const AdjArgs<T> &a, const AdjGrad<T> &gb, const AdjOut<T> &out,
                                   const ShellBox &o, const ShellBox &b, const ShellBox &gx,
                                   cudaStream_t st);
template <typename T>
cudaError_t launch_adjoint_shell_E(const AdjArgs<T> &a, const AdjSeed &sd, const AdjOut<T> &out,
                                   const ShellBox &o, const ShellBox &b, cudaStream_t st);
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
