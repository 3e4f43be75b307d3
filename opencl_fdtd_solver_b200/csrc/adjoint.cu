// Discrete adjoint of the Yee/CPML step (reverse-time sweep for ε-gradients).
//
// The forward step (yee_update.cl:11-238 as restated in yee_cell.cuh) is, for a
// lossless grid and fixed coefficients, a linear map of (E, H, ψ_E, ψ_H).  Its
// transpose is applied here in the reverse order of the forward operations:
//
//   transposed E update (k_adj_H):  for every E pair p (component c, derivative
//     axis d; ψ_E order Ex_y, Ex_z, Ey_x, Ey_z, Ez_x, Ez_y)
//       P_p' = b_e,d·P_p + s_p·ce_c·Ē_c                 (adjoint ψ recursion)
//       ḡ_p  = s_p·ce_c·ik_e,d·Ē_c + c_e,d·P_p'          (P term in the d slab only)
//       H̄   += B_d^T ḡ_p                                 (backward difference, transposed)
//   transposed H update (k_adj_E):  for every H pair p (ψ_H order Hx_y … Hz_y)
//       P_p' = b_h,d·P_p + s'_p·dtm·H̄_c
//       ā_p  = s'_p·dtm·ik_h,d·H̄_c + c_h,d·P_p'
//       Ē   += F_d^T ā_p                                 (forward difference, transposed)
//
// with s = (+,−,−,+,+,−) for the E pairs and s' = −s for the H pairs (the signs
// of each term in the forward update).  B_d zeroes index 0 and F_d the last
// index (yee_update.cl:30-35, 145-150), so
//   (B_d^T v)(x) = [x ≥ 1]·v(x) − [x ≤ n−2]·v(x+1),
//   (F_d^T v)(x) = [x ≥ 1]·v(x−1) − [x ≤ n−2]·v(x).
// P is carried in the ψ stripe layout and ping-ponged, so that a thread may read
// its neighbours' P while writing its own.
//
// ε enters through ce = dt/(ε0·ε_edge).  For ca ≡ 1, ∂E^{n+1}/∂ce = (E^{n+1} − E^n)/ce
// (the sheet term −ce·J·w of sources.cl:48 included), so the gradient box
// accumulates Σ_n Ē^{n+1}·(E^{n+1} − E^n) = ce·∂J/∂ce in float64.
//
// Compiled with --fmad=false (build.py) so that every product and sum rounds
// separately, in the order written, like the CPU restatement the tests hold it to.
#include <cuda_runtime.h>

#include <cstdint>

#include "launch_count.cuh"
#include "../../include/fdtd_b200.h"
#include "adjoint.cuh"
#include "shell_plan.cuh"

namespace fdtd {

constexpr int ADJ_TK = 32;
constexpr int ADJ_TJ = 8;

// Derivative axis of pair p (the same for the E and H orders).
__host__ __device__ constexpr int pair_axis(int p) {
    return (p == 2 || p == 4) ? 0 : ((p == 0 || p == 5) ? 1 : 2);
}
// Sign of pair p in the forward E update (+ for Ex_y, Ey_z, Ez_x).
__host__ __device__ constexpr bool pair_pos_e(int p) { return p == 0 || p == 3 || p == 4; }

template <int D>
__device__ __forceinline__ int64_t stripe_index(int i, int j, int k, int nx, int ny, int nz,
                                                int npml) {
    if (D == 0) return psi_x_index(i, j, k, nx, ny, nz, npml);
    if (D == 1) return psi_y_index(i, j, k, ny, nz, npml);
    return psi_z_index(i, j, k, ny, nz, npml);
}

// ḡ of E pair P at cell (i, j, k) with adjoint field eb and coefficient ce.
// OWN: this thread owns the cell and writes its advanced P.
template <typename T, int P, bool OWN>
__device__ __forceinline__ T e_pair(const AdjArgs<T> &a, int i, int j, int k, T eb, T ce) {
    constexpr int D = pair_axis(P);
    constexpr bool POS = pair_pos_e(P);
    const int x = D == 0 ? i : (D == 1 ? j : k);
    const int n = D == 0 ? a.nx : (D == 1 ? a.ny : a.nz);
    const T t = ce * a.cpe.ik[D][x] * eb;
    T g = POS ? t : -t;
    // the P read is issued whether or not the cell is in the slab (a harmless
    // valid address otherwise, its value discarded), so it waits behind no branch
    const bool in = in_slab(x, n, a.npml);
    const int64_t s = in ? stripe_index<D>(i, j, k, a.nx, a.ny, a.nz, a.npml) : 0;
    const T pold = *(in ? a.pe[P] + s : a.cpe.b[D]);
    if (in) {
        const T u = ce * eb;
        const T pn = a.cpe.b[D][x] * pold + (POS ? u : -u);
        if (OWN) a.pe_next[P][s] = pn;
        g = g + a.cpe.c[D][x] * pn;
    }
    return g;
}

// ā of H pair P at cell (i, j, k) with adjoint field hb.
template <typename T, int P, bool OWN>
__device__ __forceinline__ T h_pair(const AdjArgs<T> &a, int i, int j, int k, T hb) {
    constexpr int D = pair_axis(P);
    constexpr bool POS = !pair_pos_e(P);
    const int x = D == 0 ? i : (D == 1 ? j : k);
    const int n = D == 0 ? a.nx : (D == 1 ? a.ny : a.nz);
    const T t = a.dtm * a.cph.ik[D][x] * hb;
    T g = POS ? t : -t;
    const bool in = in_slab(x, n, a.npml);
    const int64_t s = in ? stripe_index<D>(i, j, k, a.nx, a.ny, a.nz, a.npml) : 0;
    const T pold = *(in ? a.ph[P] + s : a.cph.b[D]);
    if (in) {
        const T u = a.dtm * hb;
        const T pn = a.cph.b[D][x] * pold + (POS ? u : -u);
        if (OWN) a.ph_next[P][s] = pn;
        g = g + a.cph.c[D][x] * pn;
    }
    return g;
}

// Transposed E update of cell (i, j, k): H̄ += B^T ḡ(Ē, P_E) into Hout (Hout
// == a.H updates in place), P_E advanced, gradient accumulated.
template <typename T>
__device__ __forceinline__ void adj_h_cell(const AdjArgs<T> &a, const AdjGrad<T> &gb, int i,
                                           int j, int k, T *const *Hout) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int64_t sx = (int64_t)ny * nz, sy = nz;
    const int64_t idx = (int64_t)i * sx + (int64_t)j * sy + k;
    const T ex = a.E[0][idx], ey = a.E[1][idx], ez = a.E[2][idx];
    const T cx = a.ce[0][idx], cy = a.ce[1][idx], cz = a.ce[2][idx];
    const int np = a.npml;
    if (np >= 1 && i >= np && i < nx - np - 1 && j >= np && j < ny - np - 1 && k >= np &&
        k < nz - np - 1) {
        // the cell and its +1 neighbours lie in no slab: e_pair without P terms
        const T ikx = a.cpe.ik[0][i], iky = a.cpe.ik[1][j], ikz = a.cpe.ik[2][k];
        const T ikx1 = a.cpe.ik[0][i + 1], iky1 = a.cpe.ik[1][j + 1], ikz1 = a.cpe.ik[2][k + 1];
        const T g0 = cx * iky * ex, g1 = -(cx * ikz * ex), g2 = -(cy * ikx * ey);
        const T g3 = cy * ikz * ey, g4 = cz * ikx * ez, g5 = -(cz * iky * ez);
        const T g1n = -(a.ce[0][idx + 1] * ikz1 * a.E[0][idx + 1]);
        const T g3n = a.ce[1][idx + 1] * ikz1 * a.E[1][idx + 1];
        const T g0n = a.ce[0][idx + sy] * iky1 * a.E[0][idx + sy];
        const T g5n = -(a.ce[2][idx + sy] * iky1 * a.E[2][idx + sy]);
        const T g2n = -(a.ce[1][idx + sx] * ikx1 * a.E[1][idx + sx]);
        const T g4n = a.ce[2][idx + sx] * ikx1 * a.E[2][idx + sx];
        Hout[0][idx] = a.H[0][idx] + ((g3 - g3n) + (g5 - g5n));
        Hout[1][idx] = a.H[1][idx] + ((g1 - g1n) + (g4 - g4n));
        Hout[2][idx] = a.H[2][idx] + ((g0 - g0n) + (g2 - g2n));
        if (gb.active) adj_grad_cell(gb, i, j, k, ex, ey, ez);
        return;
    }
    const T g0 = e_pair<T, 0, true>(a, i, j, k, ex, cx);
    const T g1 = e_pair<T, 1, true>(a, i, j, k, ex, cx);
    const T g2 = e_pair<T, 2, true>(a, i, j, k, ey, cy);
    const T g3 = e_pair<T, 3, true>(a, i, j, k, ey, cy);
    const T g4 = e_pair<T, 4, true>(a, i, j, k, ez, cz);
    const T g5 = e_pair<T, 5, true>(a, i, j, k, ez, cz);
    T g1n = T(0), g3n = T(0), g0n = T(0), g5n = T(0), g2n = T(0), g4n = T(0);
    if (k <= nz - 2) {
        g1n = e_pair<T, 1, false>(a, i, j, k + 1, a.E[0][idx + 1], a.ce[0][idx + 1]);
        g3n = e_pair<T, 3, false>(a, i, j, k + 1, a.E[1][idx + 1], a.ce[1][idx + 1]);
    }
    if (j <= ny - 2) {
        g0n = e_pair<T, 0, false>(a, i, j + 1, k, a.E[0][idx + sy], a.ce[0][idx + sy]);
        g5n = e_pair<T, 5, false>(a, i, j + 1, k, a.E[2][idx + sy], a.ce[2][idx + sy]);
    }
    if (i <= nx - 2) {
        g2n = e_pair<T, 2, false>(a, i + 1, j, k, a.E[1][idx + sx], a.ce[1][idx + sx]);
        g4n = e_pair<T, 4, false>(a, i + 1, j, k, a.E[2][idx + sx], a.ce[2][idx + sx]);
    }
    const T tz3 = (k >= 1 ? g3 : T(0)) - g3n;
    const T ty5 = (j >= 1 ? g5 : T(0)) - g5n;
    const T tz1 = (k >= 1 ? g1 : T(0)) - g1n;
    const T tx4 = (i >= 1 ? g4 : T(0)) - g4n;
    const T ty0 = (j >= 1 ? g0 : T(0)) - g0n;
    const T tx2 = (i >= 1 ? g2 : T(0)) - g2n;
    Hout[0][idx] = a.H[0][idx] + (tz3 + ty5);
    Hout[1][idx] = a.H[1][idx] + (tz1 + tx4);
    Hout[2][idx] = a.H[2][idx] + (ty0 + tx2);
    if (gb.active) adj_grad_cell(gb, i, j, k, ex, ey, ez);
}

// Transposed H update of cell (i, j, k): Ē += F^T ā(H̄, P_H) into Eout, with H̄
// (already advanced this step) read from Hin; P_H advanced; then the seed.
template <typename T>
__device__ __forceinline__ void adj_e_cell(const AdjArgs<T> &a, const AdjSeed &sd, int i, int j,
                                           int k, T *const *Hin, T *const *Eout) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int64_t sx = (int64_t)ny * nz, sy = nz;
    const int64_t idx = (int64_t)i * sx + (int64_t)j * sy + k;
    const T hx = Hin[0][idx], hy = Hin[1][idx], hz = Hin[2][idx];
    const int np = a.npml;
    if (np >= 1 && i > np && i < nx - np && j > np && j < ny - np && k > np && k < nz - np) {
        // the cell and its -1 neighbours lie in no slab: h_pair without P terms
        const T ikx = a.cph.ik[0][i], iky = a.cph.ik[1][j], ikz = a.cph.ik[2][k];
        const T ikx1 = a.cph.ik[0][i - 1], iky1 = a.cph.ik[1][j - 1], ikz1 = a.cph.ik[2][k - 1];
        const T dm = a.dtm;
        const T a0 = -(dm * iky * hx), a1 = dm * ikz * hx, a2 = dm * ikx * hy;
        const T a3 = -(dm * ikz * hy), a4 = -(dm * ikx * hz), a5 = dm * iky * hz;
        const T a1p = dm * ikz1 * Hin[0][idx - 1];
        const T a3p = -(dm * ikz1 * Hin[1][idx - 1]);
        const T a0p = -(dm * iky1 * Hin[0][idx - sy]);
        const T a5p = dm * iky1 * Hin[2][idx - sy];
        const T a2p = dm * ikx1 * Hin[1][idx - sx];
        const T a4p = -(dm * ikx1 * Hin[2][idx - sx]);
        T ex = a.E[0][idx] + ((a3p - a3) + (a5p - a5));
        T ey = a.E[1][idx] + ((a1p - a1) + (a4p - a4));
        T ez = a.E[2][idx] + ((a0p - a0) + (a2p - a2));
        if (sd.active) add_seed<T>(sd, i, j, k, ex, ey, ez);
        Eout[0][idx] = ex;
        Eout[1][idx] = ey;
        Eout[2][idx] = ez;
        return;
    }
    const T a0 = h_pair<T, 0, true>(a, i, j, k, hx);
    const T a1 = h_pair<T, 1, true>(a, i, j, k, hx);
    const T a2 = h_pair<T, 2, true>(a, i, j, k, hy);
    const T a3 = h_pair<T, 3, true>(a, i, j, k, hy);
    const T a4 = h_pair<T, 4, true>(a, i, j, k, hz);
    const T a5 = h_pair<T, 5, true>(a, i, j, k, hz);
    T a1p = T(0), a3p = T(0), a0p = T(0), a5p = T(0), a2p = T(0), a4p = T(0);
    if (k >= 1) {
        a1p = h_pair<T, 1, false>(a, i, j, k - 1, Hin[0][idx - 1]);
        a3p = h_pair<T, 3, false>(a, i, j, k - 1, Hin[1][idx - 1]);
    }
    if (j >= 1) {
        a0p = h_pair<T, 0, false>(a, i, j - 1, k, Hin[0][idx - sy]);
        a5p = h_pair<T, 5, false>(a, i, j - 1, k, Hin[2][idx - sy]);
    }
    if (i >= 1) {
        a2p = h_pair<T, 2, false>(a, i - 1, j, k, Hin[1][idx - sx]);
        a4p = h_pair<T, 4, false>(a, i - 1, j, k, Hin[2][idx - sx]);
    }
    const T fz3 = a3p - (k <= nz - 2 ? a3 : T(0));
    const T fy5 = a5p - (j <= ny - 2 ? a5 : T(0));
    const T fz1 = a1p - (k <= nz - 2 ? a1 : T(0));
    const T fx4 = a4p - (i <= nx - 2 ? a4 : T(0));
    const T fy0 = a0p - (j <= ny - 2 ? a0 : T(0));
    const T fx2 = a2p - (i <= nx - 2 ? a2 : T(0));
    T ex = a.E[0][idx] + (fz3 + fy5);
    T ey = a.E[1][idx] + (fz1 + fx4);
    T ez = a.E[2][idx] + (fy0 + fx2);
    if (sd.active) add_seed<T>(sd, i, j, k, ex, ey, ez);
    Eout[0][idx] = ex;
    Eout[1][idx] = ey;
    Eout[2][idx] = ez;
}

// Grid-wide reverse half steps: one thread per cell (k fastest), updating
// in place (Hout = a.H, Hin = Eout... = a.E) or into separate outputs.
template <typename T>
__global__ void __launch_bounds__(ADJ_TK *ADJ_TJ)
    k_adj_H(AdjArgs<T> a, AdjGrad<T> gb, AdjOut<T> out) {
    const int k = blockIdx.x * ADJ_TK + threadIdx.x;
    const int j = blockIdx.y * ADJ_TJ + threadIdx.y;
    if (k >= a.nz || j >= a.ny) return;
    adj_h_cell<T>(a, gb, blockIdx.z, j, k, out.H);
}

template <typename T>
__global__ void __launch_bounds__(ADJ_TK *ADJ_TJ)
    k_adj_E(AdjArgs<T> a, AdjSeed sd, AdjOut<T> out) {
    const int k = blockIdx.x * ADJ_TK + threadIdx.x;
    const int j = blockIdx.y * ADJ_TJ + threadIdx.y;
    if (k >= a.nz || j >= a.ny) return;
    adj_e_cell<T>(a, sd, blockIdx.z, j, k, out.H, out.E);
}

// Shell reverse half steps: the cells of box o outside box b (shell_plan.cuh).
// Threads beyond the shell's cells accumulate the gradient of the box gx (the
// gradient box clipped to the interior march's box, whose cells the march does
// not accumulate), with the operations of adj_grad_cell.
template <typename T>
__global__ void __launch_bounds__(SHELL_THREADS)
    k_adj_shell_H(AdjArgs<T> a, AdjGrad<T> gb, AdjOut<T> out, ShellPlan sp, ShellBox gx) {
    const unsigned t = blockIdx.x * SHELL_THREADS + threadIdx.x;
    int i, j, k;
    if (shell_cell(t, sp, i, j, k)) {
        adj_h_cell<T>(a, gb, i, j, k, out.H);
        return;
    }
    const unsigned q = t - (sp.nA + sp.nB + sp.nC);
    const unsigned ez = (unsigned)(gx.hi[2] - gx.lo[2]), ey = (unsigned)(gx.hi[1] - gx.lo[1]);
    const unsigned ng = (unsigned)(gx.hi[0] - gx.lo[0]) * ey * ez;
    if (!gb.active || q >= ng) return;
    k = gx.lo[2] + (int)(q % ez);
    j = gx.lo[1] + (int)((q / ez) % ey);
    i = gx.lo[0] + (int)(q / (ez * ey));
    const int64_t idx = ((int64_t)i * a.ny + j) * a.nz + k;
    adj_grad_cell(gb, i, j, k, a.E[0][idx], a.E[1][idx], a.E[2][idx]);
}

template <typename T>
__global__ void __launch_bounds__(SHELL_THREADS)
    k_adj_shell_E(AdjArgs<T> a, AdjSeed sd, AdjOut<T> out, ShellPlan sp) {
    int i, j, k;
    if (!shell_cell(blockIdx.x * SHELL_THREADS + threadIdx.x, sp, i, j, k)) return;
    adj_e_cell<T>(a, sd, i, j, k, out.H, out.E);
}

// Seed only (before the first reverse step): one thread per patch cell.
template <typename T>
__global__ void k_adj_seed(int nx, int ny, int nz, T *E0, T *E1, T *E2, AdjSeed sd) {
    const int64_t na = sd.a1 - sd.a0, nb = sd.b1 - sd.b0;
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= na * nb) return;
    const int pa = sd.a0 + (int)(q / nb), pb = sd.b0 + (int)(q % nb);
    int i, j, k;
    if (sd.axis == 0) { i = sd.index; j = pa; k = pb; }
    else if (sd.axis == 1) { i = pa; j = sd.index; k = pb; }
    else { i = pa; j = pb; k = sd.index; }
    const int64_t idx = ((int64_t)i * ny + j) * nz + k;
    T ex = E0[idx], ey = E1[idx], ez = E2[idx];
    add_seed<T>(sd, i, j, k, ex, ey, ez);
    E0[idx] = ex;
    E1[idx] = ey;
    E2[idx] = ez;
}

// E over box [lo, hi) -> out[3][box cells]: blockIdx.y = (component, plane),
// threads over the plane's (j, k) cells, so the index arithmetic is one 32-bit
// division per thread.
template <typename T>
__global__ void k_capture(int ny, int nz, const T *E0, const T *E1, const T *E2, int3 lo,
                          int3 ext, T *out) {
    const int plane_cells = ext.y * ext.z;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= plane_cells) return;
    const int c = blockIdx.y / ext.x, ii = blockIdx.y - c * ext.x;
    const int jj = t / ext.z, kk = t - jj * ext.z;
    const int64_t idx = ((int64_t)(lo.x + ii) * ny + (lo.y + jj)) * nz + (lo.z + kk);
    const T *src = c == 0 ? E0 : (c == 1 ? E1 : E2);
    out[(int64_t)blockIdx.y * plane_cells + t] = src[idx];
}

template <typename T>
cudaError_t launch_adjoint_step(const AdjArgs<T> &a, const AdjGrad<T> &gb, const AdjSeed &sd,
                                cudaStream_t st) {
    AdjOut<T> out;
    for (int c = 0; c < 3; ++c) {
        out.E[c] = a.E[c];
        out.H[c] = a.H[c];
    }
    return launch_adjoint_grid<T>(a, gb, sd, out, st);
}

template <typename T>
cudaError_t launch_adjoint_grid(const AdjArgs<T> &a, const AdjGrad<T> &gb, const AdjSeed &sd,
                                const AdjOut<T> &out, cudaStream_t st) {
    dim3 blk(ADJ_TK, ADJ_TJ, 1);
    dim3 grd((a.nz + ADJ_TK - 1) / ADJ_TK, (a.ny + ADJ_TJ - 1) / ADJ_TJ, a.nx);
    k_adj_H<T><<<grd, blk, 0, st>>>(a, gb, out);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_adj_E<T><<<grd, blk, 0, st>>>(a, sd, out);
    count_launches(1);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_adjoint_shell_H(const AdjArgs<T> &a, const AdjGrad<T> &gb, const AdjOut<T> &out,
                                   const ShellBox &o, const ShellBox &b, const ShellBox &gx,
                                   cudaStream_t st) {
    if (!plan_fits(o)) return cudaErrorInvalidConfiguration;
    const ShellPlan sp = make_plan(o, b);
    int64_t ng = 1;
    for (int d = 0; d < 3; ++d) ng *= (gx.hi[d] > gx.lo[d]) ? gx.hi[d] - gx.lo[d] : 0;
    if (!gb.active) ng = 0;
    const uint64_t n = (uint64_t)sp.nA + sp.nB + sp.nC + (uint64_t)ng;
    if (n + SHELL_THREADS >= 0xffffffffull) return cudaErrorInvalidConfiguration;
    const unsigned nb = (unsigned)((n + SHELL_THREADS - 1) / SHELL_THREADS);
    if (nb == 0) return cudaSuccess;
    k_adj_shell_H<T><<<nb, SHELL_THREADS, 0, st>>>(a, gb, out, sp, gx);
    count_launches(1);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_adjoint_shell_E(const AdjArgs<T> &a, const AdjSeed &sd, const AdjOut<T> &out,
                                   const ShellBox &o, const ShellBox &b, cudaStream_t st) {
    if (!plan_fits(o)) return cudaErrorInvalidConfiguration;
    const ShellPlan sp = make_plan(o, b);
    const unsigned nb = shell_blocks(sp);
    if (nb == 0) return cudaSuccess;
    k_adj_shell_E<T><<<nb, SHELL_THREADS, 0, st>>>(a, sd, out, sp);
    count_launches(1);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_adjoint_seed(int nx, int ny, int nz, T *const E[3], const AdjSeed &sd,
                                cudaStream_t st) {
    const int64_t n = (int64_t)(sd.a1 - sd.a0) * (sd.b1 - sd.b0);
    if (n <= 0) return cudaSuccess;
    const int thr = 256;
    k_adj_seed<T><<<(unsigned)((n + thr - 1) / thr), thr, 0, st>>>(nx, ny, nz, E[0], E[1], E[2],
                                                                  sd);
    count_launches(1);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_capture(int ny, int nz, const T *const E[3], const int lo[3], const int hi[3],
                           T *out, cudaStream_t st) {
    const int3 l = make_int3(lo[0], lo[1], lo[2]);
    const int3 ext = make_int3(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);
    if (ext.x <= 0 || ext.y <= 0 || ext.z <= 0) return cudaSuccess;
    if (3 * (int64_t)ext.x > 65535 || (int64_t)ext.y * ext.z > 0x7fffffffLL)
        return cudaErrorInvalidValue;
    const int thr = 256;
    const dim3 grid((unsigned)(((int64_t)ext.y * ext.z + thr - 1) / thr), (unsigned)(3 * ext.x), 1);
    k_capture<T><<<grid, thr, 0, st>>>(ny, nz, E[0], E[1], E[2], l, ext, out);
    count_launches(1);
    return cudaGetLastError();
}

template cudaError_t launch_adjoint_step<float>(const AdjArgs<float> &, const AdjGrad<float> &,
                                                const AdjSeed &, cudaStream_t);
template cudaError_t launch_adjoint_step<double>(const AdjArgs<double> &,
                                                 const AdjGrad<double> &, const AdjSeed &,
                                                 cudaStream_t);
#define FDTD_ADJ_INST(T)                                                                   \
    template cudaError_t launch_adjoint_grid<T>(const AdjArgs<T> &, const AdjGrad<T> &,      \
                                                const AdjSeed &, const AdjOut<T> &,          \
                                                cudaStream_t);                               \
    template cudaError_t launch_adjoint_shell_H<T>(const AdjArgs<T> &, const AdjGrad<T> &,   \
                                                   const AdjOut<T> &, const ShellBox &,      \
                                                   const ShellBox &, const ShellBox &,       \
                                                   cudaStream_t);                            \
    template cudaError_t launch_adjoint_shell_E<T>(const AdjArgs<T> &, const AdjSeed &,      \
                                                   const AdjOut<T> &, const ShellBox &,      \
                                                   const ShellBox &, cudaStream_t);
FDTD_ADJ_INST(float)
FDTD_ADJ_INST(double)
#undef FDTD_ADJ_INST
template cudaError_t launch_adjoint_seed<float>(int, int, int, float *const[3], const AdjSeed &,
                                                cudaStream_t);
template cudaError_t launch_adjoint_seed<double>(int, int, int, double *const[3],
                                                 const AdjSeed &, cudaStream_t);
template cudaError_t launch_capture<float>(int, int, const float *const[3], const int[3],
                                           const int[3], float *, cudaStream_t);
template cudaError_t launch_capture<double>(int, int, const double *const[3], const int[3],
                                            const int[3], double *, cudaStream_t);

}  // namespace fdtd
