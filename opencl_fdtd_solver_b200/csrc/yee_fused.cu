// Fused Yee step for sm_100a: one pass over HBM for the interior of the grid.
//
// Schedule of fdtd_step (two streams):
//   side stream, forked from the caller's stream:
//   1. k_shell_H   (yee_shell.cu): H^{n+1/2} on the CPML shell outside the box
//                  B = [npml, N-npml)^3, psi_H in place, into H_next.
//   caller's stream, concurrently:
//   2. k_interior  (this file): H^{n+1/2} on B and E^{n+1} on B' = [npml+1,
//                  N-npml)^3, into H_next / E_next, sheet injections of those
//                  cells in the E epilogue.  Every H value its E stencil needs
//                  lies in B and is recomputed here, so it never waits for the
//                  shell.
//   then, after joining the side stream, E^{n+1} of every cell outside B':
//   3. k_face_E    (yee_face.cu, when npml is a multiple of 16 bytes of
//                  elements): the six CPML face slabs as TMA plane marches,
//                  with k_shell_E_boxes (yee_shell.cu) for the edges, corners
//                  and a rim row on the side stream beside it;
//   4. k_plane_dft_box (yee_shell.cu, only with plane DFT monitors): the DFTs
//                  of the monitored planes, read back from the values just
//                  written (one plane, not a field pass).
//   Otherwise 3 is k_plane_dft_box over B' and 4 is k_shell_E (yee_shell.cu),
//   one thread per shell cell with the DFTs of its cells fused.
//   FDTD_B200_SHELL_SPLIT=1 moves the shell E cells whose stencils read no H
//   of B onto the side stream behind k_shell_H (measured slower).
//
// Interior kernel.  Each CTA owns a (TJ x TK) tile of (j, k) and marches along
// i over a chunk of planes.  Plane p is brought into shared memory by TMA
// (cp.async.bulk.tensor 3-D tiled maps, no multicast) through an NSTAGE-deep
// ring completed by mbarrier transaction counts:
//   E^n(p)       rows j0-1 .. j0+TJ,  cols k0-V .. k0+TK+V-1   (V = 16 B / elem)
//   H^{n-1/2}(p) rows j0-1 .. j0+TJ-1, cols k0-V .. k0+TK-1
//   ce(p) [ca(p)] the tile only.
// Per plane the 128 "cell" threads each update V consecutive k cells (16-byte
// vector shared-memory loads and global stores) and a fifth "halo" warp
// recomputes the j0-1 row and k0-1 column of H^{n+1/2}; E^{n+1} then uses
// H^{n+1/2}(p) from shared memory and H^{n+1/2}(p-1) carried in registers.
// Interior cells need no CPML terms and no boundary guards, so the per-cell
// work is the folded-coefficient update of yee_update.cl:30-39 / 145-154.
// HBM traffic per interior cell: E, H, ce read once, E, H written once
// (60 B FP32 lossless); outputs go to separate buffers, so no CTA reads a value
// another has overwritten.
//
// Arithmetic is compiled with --fmad=false and follows the reference operand
// order, so every cell equals the split kernels and the CPU oracle bit for bit.
// Every mbarrier wait is bounded (InteriorBox::wait_polls, WAIT_LIMIT polls by
// default; fdtd_set_wait_budget lowers it); on timeout the kernel raises a
// device error flag, drains the copies it issued (with the default bound) and
// returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <array>
#include <vector>
#include <cudaTypedefs.h>

#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <unordered_map>

#include "launch_count.cuh"
#include "tma.cuh"
#include "yee_launch.cuh"

namespace fdtd {

__device__ int g_fused_error = 0;

constexpr int NSTAGE_DEFAULT = 4;  // pipeline depth (planes in flight + 2)
constexpr int NCELLTHR = 128;             // 16 vector groups x 8 rows
constexpr int NTHREADS = NCELLTHR + 32;  // + one halo warp
constexpr unsigned WAIT_LIMIT = 1u << 24;

struct alignas(64) FusedMaps {
    CUtensorMap E[3];
    CUtensorMap H[3];
    CUtensorMap C[3];
    CUtensorMap A[3];
};

// Tile of TJ rows (j) x TK cells (k): G vector groups of V cells per row.
// G = 16: 64 x 8 (FP32) / 32 x 8 (FP64); G = 8: 32 x 16 / 16 x 16, the same
// halo ratio and shared memory, chosen when it pads the k extent less.
template <typename T, int GG = 16>
struct Tile {
    static constexpr int V = 16 / (int)sizeof(T);  // elements per 16-byte vector
    static constexpr int G = GG;                    // vector groups per row
    static constexpr int TK = G * V;
    static constexpr int TJ = NCELLTHR / G;
    static constexpr int EW = TK + 2 * V, EH = TJ + 2;
    static constexpr int HW = TK + V, HH = TJ + 1;
    __host__ __device__ static constexpr int pad128(int b) { return (b + 127) / 128 * 128; }
    static constexpr int EB = pad128(EW * EH * (int)sizeof(T));
    static constexpr int HB = pad128(HW * HH * (int)sizeof(T));
    static constexpr int CB = pad128(TK * TJ * (int)sizeof(T));
    __host__ __device__ static constexpr int stage_bytes(bool lossy) {
        return 3 * EB + 3 * HB + 3 * CB * (lossy ? 2 : 1);
    }
    static constexpr int NB = 3 * HB;  // H^{n+1/2}(p) on the tile + halo, H-box layout
    __host__ __device__ static constexpr uint32_t tx_full(bool lossy) {
        return 3u * (EW * EH + HW * HH + TK * TJ * (lossy ? 2 : 1)) * sizeof(T);
    }
    __host__ __device__ static constexpr uint32_t tx_eonly() { return 3u * EW * EH * sizeof(T); }
};

// Bounded wait: false (and the device error flag set) if the phase did not
// complete within `limit` polls (the launch's InteriorBox::wait_polls,
// WAIT_LIMIT unless a caller lowered it).  A zero limit gives up at once
// unless the phase has already completed (non-blocking probe).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned limit) {
    if (limit == 0) {
        if (mbar_test_wait(bar, parity)) return true;
    } else {
        for (unsigned it = 0; it < limit; ++it)
            if (mbar_try_wait(bar, parity)) return true;
    }
    atomicOr(&g_fused_error, 1);
    return false;
}

struct InteriorBox {
    int lo[3], hi[3];  // H box B = [lo, hi); E box B' = [lo+1, hi)
    int j0base, k0base, ntk, chunk;
    unsigned wait_polls;  // budget of each pipeline wait (drains keep WAIT_LIMIT / 16)
    // dynamic shared memory layout (bytes)
    int stage_bytes, new_off, bar_off;
};

// ---------------------------------------------------------------- the kernel
template <typename T, bool LOSSY, int NSTAGE, int GG>
__global__ void __launch_bounds__(NTHREADS, 2)
    k_interior(const __grid_constant__ FusedMaps maps, const YeeArgs<T> a,
               const __grid_constant__ InteriorBox bx, const __grid_constant__ SourceList src) {
    using L = Tile<T, GG>;
    constexpr int V = L::V, TK = L::TK, TJ = L::TJ, EW = L::EW, HW = L::HW;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const int SB = bx.stage_bytes;
    T *sNew = reinterpret_cast<T *>(smem + bx.new_off);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + bx.bar_off);

    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int tile = blockIdx.x;
    const int k0 = bx.k0base + (tile % bx.ntk) * TK;
    const int j0 = bx.j0base + (tile / bx.ntk) * TJ;
    const int i0 = bx.lo[0] + blockIdx.y * bx.chunk;
    const int i1 = min(bx.hi[0], i0 + bx.chunk);
    const int pfirst = (i0 > bx.lo[0]) ? i0 - 1 : i0;  // pre-plane recomputes H(i0-1)
    const int plast = i1;                               // E only
    const int tid = threadIdx.x;
    const bool cell_thr = tid < NCELLTHR;
    const int g = tid % L::G, r = tid / L::G;  // cell threads: vector group, row

    auto sE = [&](int s, int c) {
        return reinterpret_cast<T *>(smem + s * SB + c * L::EB);
    };
    auto sH = [&](int s, int c) {
        return reinterpret_cast<T *>(smem + s * SB + 3 * L::EB + c * L::HB);
    };
    auto sC = [&](int s, int c) {
        return reinterpret_cast<T *>(smem + s * SB + 3 * L::EB + 3 * L::HB + c * L::CB);
    };
    auto sA = [&](int s, int c) {
        return reinterpret_cast<T *>(smem + s * SB + 3 * L::EB + 3 * L::HB + (3 + c) * L::CB);
    };
    auto sN = [&](int c) { return reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(sNew) + c * L::HB); };
    if (tid == 0) {
        for (int s = 0; s < NSTAGE; ++s) mbar_init(&bar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();

    int last_issued = pfirst - 1;  // thread 0 only: the last plane whose copies were issued
    auto issue = [&](int p) {
        const int s = (p - pfirst) % NSTAGE;
        last_issued = p;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (p < plast) {
            mbar_expect_tx(&bar[s], L::tx_full(LOSSY));
            for (int c = 0; c < 3; ++c) {
                tma_load_3d(sE(s, c), &maps.E[c], &bar[s], k0 - V, j0 - 1, p);
                tma_load_3d(sH(s, c), &maps.H[c], &bar[s], k0 - V, j0 - 1, p);
                tma_load_3d(sC(s, c), &maps.C[c], &bar[s], k0, j0, p);
                if (LOSSY) tma_load_3d(sA(s, c), &maps.A[c], &bar[s], k0, j0, p);
            }
        } else {
            mbar_expect_tx(&bar[s], L::tx_eonly());
            for (int c = 0; c < 3; ++c)
                tma_load_3d(sE(s, c), &maps.E[c], &bar[s], k0 - V, j0 - 1, p);
        }
    };
    if (tid == 0)
        for (int p = pfirst; p <= plast && p < pfirst + NSTAGE; ++p) issue(p);

    const T dtm_dl = a.dtm_dl, inv_dl = a.inv_dl;
    const int64_t sx = (int64_t)ny * nz;
    // cell thread geometry
    const int j = j0 + r;
    const int kb = k0 + V * g;
    const bool rowH = j >= bx.lo[1] && j < bx.hi[1];
    const bool rowE = j >= bx.lo[1] + 1 && j < bx.hi[1];
    bool kH[V], kE[V];
    bool allH = rowH, allE = rowE;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        kH[v] = (kb + v) >= bx.lo[2] && (kb + v) < bx.hi[2];
        kE[v] = (kb + v) >= bx.lo[2] + 1 && (kb + v) < bx.hi[2];
        allH = allH && kH[v];
        allE = allE && kE[v];
    }
    const int eo = (r + 1) * EW + V + V * g;  // own cells in the E box
    const int ho = (r + 1) * HW + V + V * g;  // own cells in the H / new-H box
    const int co = r * TK + V * g;            // own cells in the coefficient box

    T hyc[V], hzc[V];  // H^{n+1/2}(p-1) at own cells
#pragma unroll
    for (int v = 0; v < V; ++v) hyc[v] = hzc[v] = T(0);

    bool ok = true;
    for (int p = pfirst; p < plast; ++p) {
        const int s = (p - pfirst) % NSTAGE, s1 = (p + 1 - pfirst) % NSTAGE;
        const uint32_t par = ((p - pfirst) / NSTAGE) & 1, par1 = ((p + 1 - pfirst) / NSTAGE) & 1;
        const bool w = mbar_wait(&bar[s], par, bx.wait_polls) &&
                       mbar_wait(&bar[s1], par1, bx.wait_polls);
        if (!__syncthreads_and(w)) {  // CTA-uniform exit on a timed-out copy
            ok = false;
            break;
        }
        const bool storeH = p >= i0;
        const bool doE = p >= i0 && p >= bx.lo[0] + 1;
        const T *E0x = sE(s, 0), *E0y = sE(s, 1), *E0z = sE(s, 2);
        const T *E1y = sE(s1, 1), *E1z = sE(s1, 2);
        T ex0[V], ey0[V], ez0[V], hx[V], hy[V], hz[V];
        if (cell_thr) {
            T ezj[V], exj[V], ez1[V], ey1[V];
            ld_vec<T, V>(E0x + eo, ex0);
            ld_vec<T, V>(E0y + eo, ey0);
            ld_vec<T, V>(E0z + eo, ez0);
            ld_vec<T, V>(E0z + eo + EW, ezj);
            ld_vec<T, V>(E0x + eo + EW, exj);
            ld_vec<T, V>(E1z + eo, ez1);
            ld_vec<T, V>(E1y + eo, ey1);
            ld_vec<T, V>(sH(s, 0) + ho, hx);
            ld_vec<T, V>(sH(s, 1) + ho, hy);
            ld_vec<T, V>(sH(s, 2) + ho, hz);
            // k+1 of the last cell: first cell of the next thread in the row, or
            // the tile's halo column for the last thread
            T eyn = __shfl_down_sync(0xffffffffu, ey0[0], 1);
            T exn = __shfl_down_sync(0xffffffffu, ex0[0], 1);
            if (g == L::G - 1) {
                eyn = E0y[eo + V];
                exn = E0x[eo + V];
            }
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const T eyk = (v < V - 1) ? ey0[v + 1] : eyn;
                const T exk = (v < V - 1) ? ex0[v + 1] : exn;
                const T d_zy = ezj[v] - ez0[v], d_yz = eyk - ey0[v], d_xz = exk - ex0[v];
                const T d_zx = ez1[v] - ez0[v], d_yx = ey1[v] - ey0[v], d_xy = exj[v] - ex0[v];
                hx[v] = hx[v] - dtm_dl * (d_zy - d_yz);
                hy[v] = hy[v] - dtm_dl * (d_xz - d_zx);
                hz[v] = hz[v] - dtm_dl * (d_yx - d_xy);
            }
            st_vec<T, V>(sN(0) + ho, hx);
            st_vec<T, V>(sN(1) + ho, hy);
            st_vec<T, V>(sN(2) + ho, hz);
            if (storeH && rowH) {
                const int64_t gi = (int64_t)p * sx + (int64_t)j * nz + kb;
                if (allH) {
                    st_vec<T, V>(a.H_next[0] + gi, hx);
                    st_vec<T, V>(a.H_next[1] + gi, hy);
                    st_vec<T, V>(a.H_next[2] + gi, hz);
                } else {
#pragma unroll
                    for (int v = 0; v < V; ++v)
                        if (kH[v]) {
                            a.H_next[0][gi + v] = hx[v];
                            a.H_next[1][gi + v] = hy[v];
                            a.H_next[2][gi + v] = hz[v];
                        }
                }
            }
        } else if (doE) {
            // halo warp: H^{n+1/2} on row j0-1 (lanes 0..15) and column k0-1 (lanes 16..23)
            const int lane = tid - NCELLTHR;
            if (lane < L::G) {
                if (j0 - 1 >= bx.lo[1]) {
                    const int e = V + V * lane, h = V + V * lane;  // E box row 0, H box row 0
                    T a0[V], a1[V], a2[V], zj[V], xj[V], z1[V], y1[V], qx[V], qy[V], qz[V];
                    ld_vec<T, V>(E0x + e, a0);
                    ld_vec<T, V>(E0y + e, a1);
                    ld_vec<T, V>(E0z + e, a2);
                    ld_vec<T, V>(E0z + e + EW, zj);
                    ld_vec<T, V>(E0x + e + EW, xj);
                    ld_vec<T, V>(E1z + e, z1);
                    ld_vec<T, V>(E1y + e, y1);
                    ld_vec<T, V>(sH(s, 0) + h, qx);
                    ld_vec<T, V>(sH(s, 1) + h, qy);
                    ld_vec<T, V>(sH(s, 2) + h, qz);
                    const T yn = E0y[e + V], xn = E0x[e + V];
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        const T yk = (v < V - 1) ? a1[v + 1] : yn;
                        const T xk = (v < V - 1) ? a0[v + 1] : xn;
                        const T d_zy = zj[v] - a2[v], d_yz = yk - a1[v], d_xz = xk - a0[v];
                        const T d_zx = z1[v] - a2[v], d_yx = y1[v] - a1[v], d_xy = xj[v] - a0[v];
                        qx[v] = qx[v] - dtm_dl * (d_zy - d_yz);
                        qy[v] = qy[v] - dtm_dl * (d_xz - d_zx);
                        qz[v] = qz[v] - dtm_dl * (d_yx - d_xy);
                    }
                    st_vec<T, V>(sN(0) + h, qx);
                    st_vec<T, V>(sN(1) + h, qy);
                    st_vec<T, V>(sN(2) + h, qz);
                }
            } else if (lane < L::G + TJ) {
                const int rr = lane - L::G;
                if (k0 - 1 >= bx.lo[2] && j0 + rr < ny) {
                    const int e = (rr + 1) * EW + V - 1, h = (rr + 1) * HW + V - 1;
                    const T x0 = E0x[e], y0 = E0y[e], z0 = E0z[e];
                    const T d_zy = E0z[e + EW] - z0, d_yz = E0y[e + 1] - y0;
                    const T d_xz = E0x[e + 1] - x0, d_zx = E1z[e] - z0;
                    const T d_yx = E1y[e] - y0, d_xy = E0x[e + EW] - x0;
                    sN(0)[h] = sH(s, 0)[h] - dtm_dl * (d_zy - d_yz);
                    sN(1)[h] = sH(s, 1)[h] - dtm_dl * (d_xz - d_zx);
                    sN(2)[h] = sH(s, 2)[h] - dtm_dl * (d_yx - d_xy);
                }
            }
        }
        __syncthreads();

        T hyk0 = T(0), hxk0 = T(0);
        if (doE && cell_thr) {
            // k-1 of the first cell: last cell of the previous thread in the row,
            // or the tile's halo column for the first thread
            hyk0 = __shfl_up_sync(0xffffffffu, hy[V - 1], 1);
            hxk0 = __shfl_up_sync(0xffffffffu, hx[V - 1], 1);
            if (g == 0) {
                hyk0 = sN(1)[ho - 1];
                hxk0 = sN(0)[ho - 1];
            }
        }
        if (doE && cell_thr && rowE) {
            T hzj[V], hxj[V], cex[V], cey[V], cez[V];
            ld_vec<T, V>(sN(2) + ho - HW, hzj);
            ld_vec<T, V>(sN(0) + ho - HW, hxj);
            ld_vec<T, V>(sC(s, 0) + co, cex);
            ld_vec<T, V>(sC(s, 1) + co, cey);
            ld_vec<T, V>(sC(s, 2) + co, cez);
            T cax[V], cay[V], caz[V];
            if (LOSSY) {
                ld_vec<T, V>(sA(s, 0) + co, cax);
                ld_vec<T, V>(sA(s, 1) + co, cay);
                ld_vec<T, V>(sA(s, 2) + co, caz);
            }
            // injections: a uniform plane/tile test first, then per cell
            bool src_here = false;
            for (int q = 0; q < src.n; ++q) {
                const fdtd_source &sq = src.s[q];
                src_here |= p >= sq.i0 && p < sq.i1 && j >= sq.j0 && j < sq.j1 &&
                            sq.z >= kb && sq.z < kb + V;
            }
            if (src_here) {
#pragma unroll
                for (int v = 0; v < V; ++v) ex0[v] = apply_sources<T>(src, p, j, kb + v, ex0[v], cex[v]);
            }
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const T hyk = v ? hy[v - 1] : hyk0;
                const T hxk = v ? hx[v - 1] : hxk0;
                const T d_zy = hz[v] - hzj[v], d_yz = hy[v] - hyk, d_xz = hx[v] - hxk;
                const T d_zx = hz[v] - hzc[v], d_yx = hy[v] - hyc[v], d_xy = hx[v] - hxj[v];
                ex0[v] = (LOSSY ? cax[v] * ex0[v] : ex0[v]) + cex[v] * inv_dl * (d_zy - d_yz);
                ey0[v] = (LOSSY ? cay[v] * ey0[v] : ey0[v]) + cey[v] * inv_dl * (d_xz - d_zx);
                ez0[v] = (LOSSY ? caz[v] * ez0[v] : ez0[v]) + cez[v] * inv_dl * (d_yx - d_xy);
            }
            const int64_t gi = (int64_t)p * sx + (int64_t)j * nz + kb;
            if (allE) {
                st_vec<T, V>(a.E_next[0] + gi, ex0);
                st_vec<T, V>(a.E_next[1] + gi, ey0);
                st_vec<T, V>(a.E_next[2] + gi, ez0);
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v)
                    if (kE[v]) {
                        a.E_next[0][gi + v] = ex0[v];
                        a.E_next[1][gi + v] = ey0[v];
                        a.E_next[2][gi + v] = ez0[v];
                    }
            }
        }
        if (cell_thr) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
                hyc[v] = hy[v];
                hzc[v] = hz[v];
            }
        }
        __syncthreads();  // stage s and the new-H plane are free
        if (tid == 0 && p + NSTAGE <= plast) issue(p + NSTAGE);
    }
    if (!ok) {
        // drain: every copy issued must land before the CTA exits.  Only the
        // last NSTAGE issued planes can still be in flight (earlier ones were
        // consumed), and planes never issued are not waited for.
        __syncthreads();
        if (tid == 0) {
            const int from = max(pfirst, last_issued - NSTAGE + 1);
            for (int p = from; p <= last_issued; ++p) {
                const int s = (p - pfirst) % NSTAGE;
                const uint32_t par = ((p - pfirst) / NSTAGE) & 1;
                for (unsigned it = 0; it < WAIT_LIMIT / 16; ++it)
                    if (mbar_try_wait(&bar[s], par)) break;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- host side
namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

struct MapKey {
    const void *base;
    int nx, ny, nz, elem, b0, b1, promo;
    bool operator==(const MapKey &o) const { return memcmp(this, &o, sizeof(MapKey)) == 0; }
};
struct MapKeyHash {
    size_t operator()(const MapKey &k) const {
        size_t h = reinterpret_cast<size_t>(k.base);
        h ^= (size_t)k.nx * 1000003u ^ (size_t)k.ny * 9176u ^ (size_t)k.nz * 31u ^
             (size_t)k.b0 << 20 ^ (size_t)k.b1 << 28 ^ (size_t)k.elem;
        return h;
    }
};

std::mutex g_map_mu;
std::unordered_map<MapKey, CUtensorMap, MapKeyHash> g_maps;

}  // namespace

bool make_tensor_map(CUtensorMap *out, const void *base, int nx, int ny, int nz, int elem,
                     int b0, int b1, int l2_promote) {
    MapKey key;
    memset(&key, 0, sizeof(key));
    key.base = base;
    key.nx = nx;
    key.ny = ny;
    key.nz = nz;
    key.elem = elem;
    key.b0 = b0;
    key.b1 = b1;
    key.promo = l2_promote;
    std::lock_guard<std::mutex> lk(g_map_mu);
    auto it = g_maps.find(key);
    if (it != g_maps.end()) {
        *out = it->second;
        return true;
    }
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[3] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx};
    cuuint64_t strides[2] = {(cuuint64_t)nz * elem, (cuuint64_t)ny * nz * elem};
    cuuint32_t box[3] = {(cuuint32_t)b0, (cuuint32_t)b1, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapL2promotion promo =
        l2_promote >= 256   ? CU_TENSOR_MAP_L2_PROMOTION_L2_256B
        : l2_promote >= 128 ? CU_TENSOR_MAP_L2_PROMOTION_L2_128B
        : l2_promote >= 64  ? CU_TENSOR_MAP_L2_PROMOTION_L2_64B
                            : CU_TENSOR_MAP_L2_PROMOTION_NONE;
    CUresult r = fn(out, elem == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                    3, const_cast<void *>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, promo,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    if (g_maps.size() > 4096) g_maps.clear();
    g_maps.emplace(key, *out);
    return true;
}

namespace {

std::atomic<long long> g_wait_polls{(long long)WAIT_LIMIT};

// Pipeline depth of the interior kernel: 4 stages (2 CTAs per SM) by default;
// FDTD_B200_NSTAGE=3 selects 3 stages (3 CTAs per SM) as a tuning knob.
int stage_count() {
    static int n = [] {
        const char *v = getenv("FDTD_B200_NSTAGE");
        return (v && atoi(v) == 3) ? 3 : NSTAGE_DEFAULT;
    }();
    return n;
}

// Chunks along i: whole waves of resident CTAs, chunks of at least 16 planes
// (8 when there are fewer tiles than resident CTA slots: a small grid needs
// the shorter marches to fill the GPU, at one extra plane read per chunk).
int choose_chunks(int tiles, int nplanes, int sms) {
    const int slots = (stage_count() == 3 ? 3 : 2) * sms;
    const int min_len = tiles < slots ? 8 : 16;
    int best = 1;
    double best_score = -1.0;
    for (int c = 1; c <= 64; ++c) {
        const int len = (nplanes + c - 1) / c;
        if (len < min_len && c > 1) break;
        const double waves = (double)tiles * c / slots;
        const double fill = waves / std::ceil(waves);
        const double score = fill * (1.0 - 1.0 / (len + 1.0));
        if (score > best_score + 1e-9) {
            best_score = score;
            best = c;
        }
    }
    return best;
}

template <typename T, int GG>
bool build_maps(const YeeArgs<T> &a, FusedMaps &maps) {
    using L = Tile<T, GG>;
    const int elem = (int)sizeof(T);
    // the maps of this buffer set, built once
    static KeyedCache<FusedMaps, 16> cache;
    uint64_t key[16];
    for (int c = 0; c < 3; ++c) {
        key[c] = (uint64_t)(uintptr_t)a.E[c];
        key[3 + c] = (uint64_t)(uintptr_t)a.H[c];
        key[6 + c] = (uint64_t)(uintptr_t)a.ce[c];
        key[9 + c] = a.lossy ? (uint64_t)(uintptr_t)a.ca[c] : 0;
    }
    key[12] = (uint64_t)a.nx;
    key[13] = (uint64_t)a.ny;
    key[14] = (uint64_t)a.nz;
    key[15] = (uint64_t)(a.lossy != 0);
    if (cache.get(key, maps)) return true;
    memset(&maps, 0, sizeof(maps));
    for (int c = 0; c < 3; ++c) {
        if (!make_tensor_map(&maps.E[c], a.E[c], a.nx, a.ny, a.nz, elem, L::EW, L::EH) ||
            !make_tensor_map(&maps.H[c], a.H[c], a.nx, a.ny, a.nz, elem, L::HW, L::HH) ||
            !make_tensor_map(&maps.C[c], a.ce[c], a.nx, a.ny, a.nz, elem, L::TK, L::TJ))
            return false;
        if (a.lossy && !make_tensor_map(&maps.A[c], a.ca[c], a.nx, a.ny, a.nz, elem, L::TK, L::TJ))
            return false;
    }
    cache.put(key, maps);
    return true;
}

template <typename T, int GG>
cudaError_t launch_interior(const YeeArgs<T> &a, const FusedMaps &maps, const ShellBox &hb,
                            const SourceList &src, cudaStream_t st) {
    using L = Tile<T, GG>;
    InteriorBox bx;
    for (int d = 0; d < 3; ++d) {
        bx.lo[d] = hb.lo[d];
        bx.hi[d] = hb.hi[d];
    }
    bx.k0base = (hb.lo[2] / L::V) * L::V;  // TMA x coordinates stay 16-byte aligned
    bx.j0base = hb.lo[1];
    bx.ntk = (hb.hi[2] - bx.k0base + L::TK - 1) / L::TK;
    const int ntj = (hb.hi[1] - bx.j0base + L::TJ - 1) / L::TJ;
    const int tiles = bx.ntk * ntj;
    const int sms = device_sm_count();
    const int nplanes = hb.hi[0] - hb.lo[0];
    const int nchunk = choose_chunks(tiles, nplanes, sms);
    bx.chunk = (nplanes + nchunk - 1) / nchunk;
    dim3 grid(tiles, (nplanes + bx.chunk - 1) / bx.chunk, 1);
    bx.stage_bytes = L::stage_bytes(a.lossy != 0);
    bx.wait_polls = (unsigned)g_wait_polls.load();
    const int nstage = stage_count();
    bx.new_off = nstage * bx.stage_bytes;
    bx.bar_off = bx.new_off + L::NB;
    const size_t smem = bx.bar_off + 64 + 128;
    cudaError_t e = cudaSuccess;
#define FDTD_LAUNCH_INTERIOR(LS, NS)                                                           \
    do {                                                                                       \
        e = ensure_max_dynamic_smem((const void *)k_interior<T, LS, NS, GG>, (int)smem);       \
        if (e != cudaSuccess) return e;                                                        \
        k_interior<T, LS, NS, GG><<<grid, NTHREADS, smem, st>>>(maps, a, bx, src);             \
        count_launches(1);                                                                     \
    } while (0)
    if (a.lossy) {
        if (nstage == 3) FDTD_LAUNCH_INTERIOR(true, 3);
        else FDTD_LAUNCH_INTERIOR(true, 4);
    } else {
        if (nstage == 3) FDTD_LAUNCH_INTERIOR(false, 3);
        else FDTD_LAUNCH_INTERIOR(false, 4);
    }
#undef FDTD_LAUNCH_INTERIOR
    return cudaGetLastError();
}

}  // namespace

// ---- per-launch timing of the step (diagnostics) ---------------------------
namespace {
constexpr int NEV = 7;
constexpr int NPROF = 5;
struct StepProfiler {
    std::mutex mu;
    bool on = false;
    std::vector<std::array<cudaEvent_t, NEV>> pending;
    std::vector<bool> dft_last;  // per pending step: the plane DFT ran after shell E
    double ms[NPROF] = {0.0, 0.0, 0.0, 0.0, 0.0};
    int steps = 0;
};
StepProfiler g_prof;

// Waits for the recorded steps, adds their launch times, releases the events.
cudaError_t prof_flush_locked() {
    cudaError_t err = cudaSuccess;
    for (size_t q = 0; q < g_prof.pending.size(); ++q) {
        auto &ev = g_prof.pending[q];
        // ev: 0 start, 1 shell H done (side stream), 2 outer shell E done (side),
        // 3 interior done, 4 joined, 5 plane DFT done, 6 rim E done; with the
        // face kernels 5 is shell E done and 6 plane DFT done
        cudaError_t e = cudaEventSynchronize(ev[6]);
        const bool late = g_prof.dft_last[q];
        const int from[NPROF] = {0, 1, 0, late ? 5 : 4, late ? 4 : 5};
        const int to[NPROF] = {1, 2, 3, late ? 6 : 5, late ? 5 : 6};
        for (int s = 0; s < NPROF && e == cudaSuccess; ++s) {
            float t = 0.f;
            e = cudaEventElapsedTime(&t, ev[from[s]], ev[to[s]]);
            g_prof.ms[s] += t;
        }
        if (e != cudaSuccess) err = e;
        for (cudaEvent_t x : ev) cudaEventDestroy(x);
        ++g_prof.steps;
    }
    g_prof.pending.clear();
    g_prof.dft_last.clear();
    return err;
}

bool prof_begin(std::array<cudaEvent_t, NEV> &ev) {
    std::lock_guard<std::mutex> lk(g_prof.mu);
    if (!g_prof.on) return false;
    for (int s = 0; s < NEV; ++s)
        if (cudaEventCreate(&ev[s]) != cudaSuccess) {
            for (int q = 0; q < s; ++q) cudaEventDestroy(ev[q]);
            return false;
        }
    return true;
}

void prof_end(const std::array<cudaEvent_t, NEV> &ev, bool dft_last) {
    std::lock_guard<std::mutex> lk(g_prof.mu);
    g_prof.pending.push_back(ev);
    g_prof.dft_last.push_back(dft_last);
    if (g_prof.pending.size() >= 2048) prof_flush_locked();
}
}  // namespace

// Side stream (per host thread, device and slot) on which the CPML-shell H
// kernel and the outer shell-E kernel run concurrently with the interior
// kernel: they are independent of it (the interior kernel recomputes every H it
// needs from E and H, and the outer E cells read no H of the interior box), so
// the latency-bound shell fills the bandwidth the interior kernel leaves.
// Joined back to the caller's stream by an event before the rim E cells.
namespace {
thread_local std::unordered_map<int, SideStream> t_side;
}

int device_sm_count() {
    static std::atomic<int> sms[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    int v = sms[dev].load();
    if (v <= 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            v <= 0)
            return 148;
        sms[dev].store(v);
    }
    return v;
}

// Reads the function's current limit (per context, so a device reset that
// restores the default is seen) and raises it only when it is too low.
cudaError_t ensure_max_dynamic_smem(const void *func, int bytes) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, func);
    if (e != cudaSuccess) return e;
    if (fa.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
    return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

cudaError_t side_stream(SideStream **out, int slot) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const int key = dev * 4 + (slot & 3);
    auto it = t_side.find(key);
    if (it == t_side.end()) {
        SideStream ss;
        // FDTD_B200_SIDE_PRIO=1 gives the side stream the device's highest
        // priority (its blocks are dispatched before the interior kernel's)
        int lo = 0, hi = 0;
        const char *pv = getenv("FDTD_B200_SIDE_PRIO");
        const bool prio = pv && atoi(pv) == 1 && cudaDeviceGetStreamPriorityRange(&lo, &hi) ==
                                                      cudaSuccess;
        if ((e = cudaStreamCreateWithPriority(&ss.s, cudaStreamNonBlocking, prio ? hi : 0)) !=
            cudaSuccess)
            return e;
        if ((e = cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&ss.join, cudaEventDisableTiming)) != cudaSuccess)
            return e;
        it = t_side.emplace(key, ss).first;
    }
    *out = &it->second;
    return cudaSuccess;
}

void profile_enable(bool on) {
    std::lock_guard<std::mutex> lk(g_prof.mu);
    if (on) {
        prof_flush_locked();
        for (double &m : g_prof.ms) m = 0.0;
        g_prof.steps = 0;
    }
    g_prof.on = on;
}

cudaError_t profile_read(double ms[5], int *steps) {
    std::lock_guard<std::mutex> lk(g_prof.mu);
    cudaError_t e = prof_flush_locked();
    for (int s = 0; s < NPROF; ++s) ms[s] = g_prof.ms[s];
    *steps = g_prof.steps;
    return e;
}

// FDTD_B200_SHELL_SPLIT=1 splits the shell E cells whose stencils read no H of
// B off onto the side stream, behind k_shell_H (measured slower at 512³: the
// side stream is starved while the interior kernel holds the SMs, 2.05 against
// 1.88 ms); by default all shell E cells run after the join.
bool split_shell_e() {
    static const bool v = [] {
        const char *e = getenv("FDTD_B200_SHELL_SPLIT");
        return e && atoi(e) == 1;
    }();
    return v;
}

template <typename T>
cudaError_t launch_step_fused(const YeeArgs<T> &a, const SourceList &src, const PlaneList &pl,
                              cudaStream_t st) {
    const int elem = (int)sizeof(T);
    const int n[3] = {a.nx, a.ny, a.nz};
    // interior H box B = [npml, N-npml)^3 (x on a slab: [pml_lo, nx - pml_hi -
    // ghost_hi), so the upper ghost plane, whose forward differences would read
    // past the slab, is left to the boundary-guarded shell kernel); the fused
    // kernel needs npml >= 1, a box of at least two cells per axis and
    // TMA-compatible (16-byte) strides and base addresses
    int blo[3], bhi[3];
    for (int d = 0; d < 3; ++d) {
        blo[d] = a.npml;
        bhi[d] = n[d] - a.npml;
    }
    blo[0] = a.xb.pml_lo;
    bhi[0] = n[0] - a.xb.pml_hi - a.ghost_hi;
    bool use_interior = a.npml >= 1 && ((int64_t)a.nz * elem) % 16 == 0;
    for (int d = 0; d < 3; ++d) use_interior = use_interior && bhi[d] - blo[d] >= 2;
    for (int c = 0; c < 3 && use_interior; ++c) {
        const void *ptrs[5] = {a.E[c], a.H[c], a.ce[c], a.E_next[c], a.H_next[c]};
        for (const void *q : ptrs)
            if (reinterpret_cast<uintptr_t>(q) % 16 != 0) use_interior = false;
        if (a.lossy && reinterpret_cast<uintptr_t>(a.ca[c]) % 16 != 0) use_interior = false;
    }
    // tile shape: the one that pads the interior's k extent [lo, hi) least
    // (k0 starts at lo rounded down to a 16-byte boundary)
    int gsel = 16;
    {
        const int k0 = (blo[2] / Tile<T, 16>::V) * Tile<T, 16>::V, ext = bhi[2] - k0;
        const int w16 = Tile<T, 16>::TK, w8 = Tile<T, 8>::TK;
        // 64 x 8 streams better (measured at 512³: 1.18 ms against 1.31 ms for the
        // 32 x 16 tile, which pads 480 cells to 480 instead of 512); the 32 x 16
        // tile is taken only where it saves a fifth of the padded k extent
        if (5 * ((ext + w16 - 1) / w16 * w16) > 6 * ((ext + w8 - 1) / w8 * w8)) gsel = 8;
    }
    FusedMaps maps;
    if (use_interior && !(gsel == 8 ? build_maps<T, 8>(a, maps) : build_maps<T, 16>(a, maps)))
        use_interior = false;
    // hbox = B (H of the interior kernel), ebox = B' (its E), rbox = [lo, hi+1):
    // the E cells outside rbox read no H of B, the rim rbox \ B' does
    ShellBox hbox, ebox, rbox, none, all;
    for (int d = 0; d < 3; ++d) {
        all.lo[d] = 0;
        all.hi[d] = n[d];
        hbox.lo[d] = use_interior ? blo[d] : 0;
        hbox.hi[d] = use_interior ? bhi[d] : 0;
        ebox.lo[d] = use_interior ? blo[d] + 1 : 0;
        ebox.hi[d] = use_interior ? bhi[d] : 0;
        rbox.lo[d] = use_interior ? blo[d] : 0;
        rbox.hi[d] = use_interior ? bhi[d] + 1 : n[d];
        none.lo[d] = none.hi[d] = 0;
    }
    SideStream *side = nullptr;
    if (use_interior) {
        cudaError_t e = side_stream(&side);
        if (e != cudaSuccess) return e;
    }
    std::array<cudaEvent_t, NEV> ev;
    const bool prof = prof_begin(ev);
    if (prof) cudaEventRecord(ev[0], st);
    cudaError_t e = cudaSuccess;
    if (use_interior) {
        // shell H, then the outer shell E, on the side stream, concurrent with
        // the interior kernel
        if ((e = cudaEventRecord(side->fork, st)) == cudaSuccess &&
            (e = cudaStreamWaitEvent(side->s, side->fork, 0)) == cudaSuccess)
            e = launch_shell_H<T>(a, hbox, side->s);
        if (prof) cudaEventRecord(ev[1], side->s);
        if (e == cudaSuccess && split_shell_e())
            e = launch_shell_E_region<T>(a, all, rbox, src, pl, side->s);
        if (prof) cudaEventRecord(ev[2], side->s);
        cudaError_t e2 = cudaEventRecord(side->join, side->s);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess)
            e = gsel == 8 ? launch_interior<T, 8>(a, maps, hbox, src, st)
                          : launch_interior<T, 16>(a, maps, hbox, src, st);
        if (prof) cudaEventRecord(ev[3], st);
        e2 = cudaStreamWaitEvent(st, side->join, 0);
        if (e == cudaSuccess) e = e2;
    } else {
        e = launch_shell_H<T>(a, none, st);
        if (prof) {
            cudaEventRecord(ev[1], st);
            cudaEventRecord(ev[2], st);
            cudaEventRecord(ev[3], st);
        }
    }
    if (prof) cudaEventRecord(ev[4], st);
    bool faces = use_interior && !split_shell_e() && face_path_ok<T>(a);
    if (faces && e == cudaSuccess) {
        // shell E through the CPML face marches, then the plane DFTs of every
        // monitored cell in one pass over the planes
        e = launch_shell_E_faces<T>(a, src, st, side);
        if (e == cudaErrorNotSupported) {
            faces = false;  // no tensor maps: the per-cell shell E below
            e = cudaSuccess;
        }
    }
    if (faces) {
        if (prof) cudaEventRecord(ev[5], st);
        if (e == cudaSuccess && pl.n) e = launch_plane_dft_box<T>(a, all, pl, st);
    } else {
        // plane DFTs of the cells the interior kernel updated
        if (e == cudaSuccess && use_interior && pl.n)
            e = launch_plane_dft_box<T>(a, ebox, pl, st);
        if (prof) cudaEventRecord(ev[5], st);
        // E of the rim (or of the whole grid without an interior box), or of
        // every cell outside B' when the outer part did not run on the side
        // stream, with the DFTs of those cells
        if (e == cudaSuccess)
            e = launch_shell_E_region<T>(a, (use_interior && split_shell_e()) ? rbox : all, ebox,
                                         src, pl, st);
    }
    if (prof) {
        cudaEventRecord(ev[6], st);
        prof_end(ev, faces);
    }
    return e;
}

template cudaError_t launch_step_fused<float>(const YeeArgs<float> &, const SourceList &,
                                              const PlaneList &, cudaStream_t);
template cudaError_t launch_step_fused<double>(const YeeArgs<double> &, const SourceList &,
                                               const PlaneList &, cudaStream_t);

unsigned interior_wait_polls() { return (unsigned)g_wait_polls.load(); }
int interior_chunks(int tiles, int nplanes, int sms) { return choose_chunks(tiles, nplanes, sms); }

void set_interior_wait_polls(int64_t polls) {
    g_wait_polls.store(polls < 0 ? (long long)WAIT_LIMIT
                                 : (long long)(polls > (int64_t)WAIT_LIMIT ? WAIT_LIMIT : polls));
}

// The interior kernel's and the face kernels' flags (one status bit).
int read_fused_error(int reset) {
    const int f = read_face_error(reset);
    int v = 0;
    cudaMemcpyFromSymbol(&v, g_fused_error, sizeof(int));
    if (reset) {
        int z = 0;
        cudaMemcpyToSymbol(g_fused_error, &z, sizeof(int));
    }
    return v | f;
}

}  // namespace fdtd
