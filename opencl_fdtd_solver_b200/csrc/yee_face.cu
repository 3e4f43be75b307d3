// CPML shell E half step as plane marches over the CPML face slabs (sm_100a).
//
// Once the interior kernel and k_shell_H have written H^{n+1/2} (H_next) on
// the whole grid, E^{n+1} of the cells outside the interior E box B' =
// [npml+1, N-npml)^3 remains.  Almost all of them lie in exactly one CPML slab
// and need only that axis' ψ_E pair (P = npml, I = [P+1, N-P)):
//   face x: i in [0, P] or [N-P, N),  j, k in [P, N-P)
//           (the plane i = P is the interior-formula rim just below B')
//   face y: i in I,  j in [0, P) or [N-P, N),  k in [P, N-P)
//   face z: i, j in I,  k in [0, P] or [N-P, N)
//           (the column k = P is the interior-formula rim)
// Each CTA owns a (TJ x TK) tile of (j, k) of one face region and marches
// along i over a chunk of planes.  Per plane one thread issues TMA 3-D tiled
// loads (cp.async.bulk.tensor, no multicast) into an NSTAGE-deep ring of
// stages completed by mbarrier transaction counts:
//   H^{n+1/2}(p)  rows j0-1 .. j0+TJ-1, cols k0-V .. k0+TK-1 (the j-1 row and
//                 k-1 column of the stencil; V = 16 B / elem)
//   E^n(p), ce(p) [ca(p)], and the face axis' ψ_E pair on the tile.
// H^{n+1/2}(p-1) of the own cells is carried in registers from the previous
// plane (a chunk starts with one H-only plane).  The threads each update V
// consecutive k cells with 16-byte shared-memory loads and global stores; ψ_E
// is read through the stage and written back in place (each cell by one CTA).
// Plane DFTs are not accumulated here: a global read-modify-write inside the
// march would hold every warp of the CTA at the plane barrier, so the fused
// step accumulates the monitored planes in one pass after the shell E kernels.
//
// The remaining shell E cells (edges and corners where two slabs overlap and
// the rim row j = P of the I planes) go to the per-cell kernel
// k_shell_E_boxes, on the side stream, concurrently.
//
// Arithmetic is e_cell's (yee_cell.cuh, reference yee_update.cl:145-154,
// 195-237) with the ψ terms of the other axes zero, compiled with --fmad=false,
// so every cell rounds exactly as in the per-cell kernels and the CPU oracle.
// Every mbarrier wait is bounded by the interior kernel's wait budget; on a
// timeout the CTA raises the fused-step error flag, drains the copies it
// issued and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "launch_count.cuh"
#include "shell_plan.cuh"
#include "tma.cuh"
#include "yee_launch.cuh"

namespace fdtd {

__device__ int g_face_error = 0;

namespace {

constexpr int FACE_THREADS = 128;
constexpr int FACE_NSTAGE = 4;
constexpr unsigned FACE_DRAIN_LIMIT = 1u << 20;
constexpr int FACE_MAX_CHUNK = 64;  // planes per CTA (per-plane coefficients in shared memory)

// Tile of TJ rows (j) x TK cells (k): G vector groups of V cells per row.
// x and y faces: 64 x 8 (FP32) / 32 x 8 (FP64); z faces: 20 x 25 / 10 x 25
// (125 of the 128 threads), whose k extent holds a 16-cell CPML slab and its
// rim column.
template <typename T, int AX>
struct FaceTile {
    static constexpr int V = 16 / (int)sizeof(T);
    static constexpr int G = (AX == 2) ? 5 : 16;
    static constexpr int TK = G * V;
    static constexpr int TJ = (AX == 2) ? 25 : FACE_THREADS / G;
    static constexpr int HW = TK + V, HH = TJ + 1;
    __host__ __device__ static constexpr int pad128(int b) { return (b + 127) / 128 * 128; }
    static constexpr int HB = pad128(HW * HH * (int)sizeof(T));
    static constexpr int CB = pad128(TK * TJ * (int)sizeof(T));
    __host__ __device__ static constexpr int stage_bytes(bool lossy) {
        return 3 * HB + (3 + 3 + (lossy ? 3 : 0) + 2) * CB;
    }
    __host__ __device__ static constexpr uint32_t tx_h() {
        return 3u * (uint32_t)(HW * HH * sizeof(T));
    }
    __host__ __device__ static constexpr uint32_t tx_cells(bool lossy, bool psi) {
        return (uint32_t)((6 + (lossy ? 3 : 0) + (psi ? 2 : 0)) * TK * TJ * sizeof(T));
    }
};

// Tensor maps by tile shape: [0] the x/y-face tile, [1] the z-face tile; P
// per face: its ψ_E pair (x: Ey_x, Ez_x; y: Ex_y, Ez_y; z: Ex_z, Ey_z).
struct alignas(64) FaceMaps {
    CUtensorMap H[2][3], E[2][3], C[2][3], A[2][3];
    CUtensorMap P[3][2];
};

// One face: its low (r = 0) and high (r = 1) region [lo, hi) with ntj x
// ntk[r] tiles and nchunk chunks of `chunk` planes along i; CTAs [first,
// first + ctas) of the launch.
struct FaceBox {
    int lo[2][3], hi[2][3];
    int ntj, ntk[2], nchunk, chunk;
    int first, ctas;
};

struct FaceSet {
    FaceBox f[3];
    unsigned wait_polls;
    int stage_bytes, bar_off;
};

__device__ __forceinline__ bool face_wait(uint64_t *bar, uint32_t parity, unsigned limit) {
    if (limit == 0) {
        if (mbar_test_wait(bar, parity)) return true;
    } else {
        for (unsigned it = 0; it < limit; ++it)
            if (mbar_try_wait(bar, parity)) return true;
    }
    atomicOr(&g_face_error, 1);
    return false;
}

template <typename T, bool LOSSY, int NSTAGE, int AX>
__device__ __forceinline__ void face_march(const FaceMaps &maps, const YeeArgs<T> &a,
                                           const FaceSet &fs, const SourceList &src,
                                           unsigned char *smem, int b) {
    using L = FaceTile<T, AX>;
    constexpr int V = L::V, TK = L::TK, TJ = L::TJ, HW = L::HW, G = L::G;
    constexpr int SH = (AX == 2) ? 1 : 0;
    const FaceBox &f = fs.f[AX];
    const int cidx = b % f.nchunk, t = b / f.nchunk;
    const int per0 = f.ntj * f.ntk[0];
    const int r = t < per0 ? 0 : 1, tt = t - r * per0;
    const int k0 = f.lo[r][2] + (tt % f.ntk[r]) * TK;
    const int j0 = f.lo[r][1] + (tt / f.ntk[r]) * TJ;
    const int i0 = f.lo[r][0] + cidx * f.chunk;
    const int i1 = min(f.hi[r][0], i0 + f.chunk);
    if (i0 >= i1) return;  // CTA-uniform, before any barrier
    const int pfirst = (i0 > 0) ? i0 - 1 : i0;  // H-only plane for H(i0-1)

    const int nx = a.nx, ny = a.ny, nz = a.nz, npml = a.npml;
    const int SB = fs.stage_bytes;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + fs.bar_off);
    auto sH = [&](int s, int c) { return reinterpret_cast<T *>(smem + s * SB + c * L::HB); };
    auto sE = [&](int s, int c) {
        return reinterpret_cast<T *>(smem + s * SB + 3 * L::HB + c * L::CB);
    };
    auto sC = [&](int s, int c) {
        return reinterpret_cast<T *>(smem + s * SB + 3 * L::HB + (3 + c) * L::CB);
    };
    auto sA = [&](int s, int c) {
        return reinterpret_cast<T *>(smem + s * SB + 3 * L::HB + (6 + c) * L::CB);
    };
    auto sP = [&](int s, int c) {
        return reinterpret_cast<T *>(smem + s * SB + 3 * L::HB + ((LOSSY ? 9 : 6) + c) * L::CB);
    };
    const int tid = threadIdx.x;
    // per-plane CPML coefficients of the x axis for the chunk's planes
    T *s_ik = reinterpret_cast<T *>(smem + fs.bar_off + 64);
    T *s_b = s_ik + FACE_MAX_CHUNK, *s_c = s_b + FACE_MAX_CHUNK;
    for (int q = tid; q < i1 - i0; q += FACE_THREADS) {
        s_ik[q] = a.cpe.ik[0][i0 + q];
        s_b[q] = a.cpe.b[0][i0 + q];
        s_c[q] = a.cpe.c[0][i0 + q];
    }
    if (tid == 0) {
        for (int s = 0; s < NSTAGE; ++s) mbar_init(&bar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();

    // the x faces' plane i = P is the interior-formula rim: no ψ
    auto psi_plane = [&](int p) { return AX != 0 || p < npml || p >= nx - npml; };
    int last_issued = pfirst - 1;  // thread 0 only
    auto issue = [&](int p) {
        const int s = (p - pfirst) % NSTAGE;
        last_issued = p;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (p < i0) {
            mbar_expect_tx(&bar[s], L::tx_h());
            for (int c = 0; c < 3; ++c)
                tma_load_3d(sH(s, c), &maps.H[SH][c], &bar[s], k0 - V, j0 - 1, p);
            return;
        }
        const bool ps = psi_plane(p);
        mbar_expect_tx(&bar[s], L::tx_h() + L::tx_cells(LOSSY, ps));
        for (int c = 0; c < 3; ++c) {
            tma_load_3d(sH(s, c), &maps.H[SH][c], &bar[s], k0 - V, j0 - 1, p);
            tma_load_3d(sE(s, c), &maps.E[SH][c], &bar[s], k0, j0, p);
            tma_load_3d(sC(s, c), &maps.C[SH][c], &bar[s], k0, j0, p);
            if (LOSSY) tma_load_3d(sA(s, c), &maps.A[SH][c], &bar[s], k0, j0, p);
        }
        if (ps) {
            int c0, c1, c2;
            if (AX == 0) {
                c0 = k0;
                c1 = j0;
                c2 = pml_layer(p, nx, npml);
            } else if (AX == 1) {
                c0 = k0;
                c1 = pml_layer(j0, ny, npml);
                c2 = p;
            } else {
                // layer of the tile's first cell by region (a low tile that
                // starts at the rim column reads high layers it does not use)
                c0 = (r == 0) ? k0 : npml + k0 - (nz - npml);
                c1 = j0;
                c2 = p;
            }
            tma_load_3d(sP(s, 0), &maps.P[AX][0], &bar[s], c0, c1, c2);
            tma_load_3d(sP(s, 1), &maps.P[AX][1], &bar[s], c0, c1, c2);
        }
    };
    if (tid == 0)
        for (int p = pfirst; p < i1 && p < pfirst + NSTAGE; ++p) issue(p);

    // own cells: row j, V cells from kb (the idle threads of the z-face tile
    // have no row and point at row 0 of the tiles)
    const int g = tid % G, rr = tid / G;
    const int j = j0 + rr, kb = k0 + V * g;
    const bool rowv = rr < TJ && j < f.hi[r][1];
    bool kv[V];
    bool allv = rowv;
#pragma unroll
    for (int v = 0; v < V; ++v) {
        kv[v] = rowv && kb + v < f.hi[r][2];
        allv = allv && kv[v];
    }
    const int ho = ((rr < TJ ? rr : 0) + 1) * HW + V + V * g;  // own cells in the H box
    const int co = (rr < TJ ? rr : 0) * TK + V * g;            // own cells in the cell tiles
    // the z-face group holding the rim column k = P: its first cell takes the
    // interior formula and has no ψ (P is a multiple of V, the others are masked)
    const bool rim_group = AX == 2 && kb == npml;
    const Cpml1D<T> &cp = a.cpe;
    const T iky = rowv ? cp.ik[1][j] : T(0);
    T ikz[V], bz[V], cz[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        ikz[v] = kv[v] ? cp.ik[2][kb + v] : T(0);
        bz[v] = (AX == 2 && kv[v]) ? cp.b[2][kb + v] : T(0);
        cz[v] = (AX == 2 && kv[v]) ? cp.c[2][kb + v] : T(0);
    }
    const T by = (AX == 1 && rowv) ? cp.b[1][j] : T(0);
    const T cy = (AX == 1 && rowv) ? cp.c[1][j] : T(0);
    // sheet injections that can reach the own cells (row and k range; the
    // plane range is tested per cell by apply_sources)
    bool src_row = false;
    for (int q = 0; q < src.n; ++q) {
        const fdtd_source &sq = src.s[q];
        src_row |= rowv && j >= sq.j0 && j < sq.j1 && sq.z >= kb && sq.z < kb + V;
    }
    T *const qa = a.psi_e[AX == 0 ? 2 : (AX == 1 ? 0 : 1)];
    T *const qb = a.psi_e[AX == 0 ? 4 : (AX == 1 ? 5 : 3)];
    const int64_t sx = (int64_t)ny * nz;

    T hyc[V], hzc[V];  // H^{n+1/2}(p-1) at the own cells
#pragma unroll
    for (int v = 0; v < V; ++v) hyc[v] = hzc[v] = T(0);

    bool ok = true;
    for (int p = pfirst; p < i1; ++p) {
        const int s = (p - pfirst) % NSTAGE;
        const uint32_t par = ((p - pfirst) / NSTAGE) & 1;
        const bool w = face_wait(&bar[s], par, fs.wait_polls);
        if (!__syncthreads_and(w)) {  // CTA-uniform exit on a timed-out copy
            ok = false;
            break;
        }
        T hx[V], hy[V], hz[V];
        ld_vec<T, V>(sH(s, 0) + ho, hx);
        ld_vec<T, V>(sH(s, 1) + ho, hy);
        ld_vec<T, V>(sH(s, 2) + ho, hz);
        if (p >= i0 && rowv) {
            const bool ps = psi_plane(p);
            T hzj[V], hxj[V], ex[V], ey[V], ez[V], cex[V], cey[V], cez[V];
            T cax[V], cay[V], caz[V], pa[V], pb[V];
            ld_vec<T, V>(sH(s, 2) + ho - HW, hzj);
            ld_vec<T, V>(sH(s, 0) + ho - HW, hxj);
            const T hyk0 = sH(s, 1)[ho - 1], hxk0 = sH(s, 0)[ho - 1];
            ld_vec<T, V>(sE(s, 0) + co, ex);
            ld_vec<T, V>(sE(s, 1) + co, ey);
            ld_vec<T, V>(sE(s, 2) + co, ez);
            ld_vec<T, V>(sC(s, 0) + co, cex);
            ld_vec<T, V>(sC(s, 1) + co, cey);
            ld_vec<T, V>(sC(s, 2) + co, cez);
            if (LOSSY) {
                ld_vec<T, V>(sA(s, 0) + co, cax);
                ld_vec<T, V>(sA(s, 1) + co, cay);
                ld_vec<T, V>(sA(s, 2) + co, caz);
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) cax[v] = cay[v] = caz[v] = T(1);
            }
            if (ps) {
                ld_vec<T, V>(sP(s, 0) + co, pa);
                ld_vec<T, V>(sP(s, 1) + co, pb);
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v) pa[v] = pb[v] = T(0);
            }
            // sheet injections on E^n (apply_sources tests each cell)
            if (src_row) {
#pragma unroll
                for (int v = 0; v < V; ++v)
                    if (kv[v]) ex[v] = apply_sources<T>(src, p, j, kb + v, ex[v], cex[v]);
            }
            const T ikx = s_ik[p - i0];
            const T bx = (AX == 0 && ps) ? s_b[p - i0] : T(0);
            const T cx = (AX == 0 && ps) ? s_c[p - i0] : T(0);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int k = kb + v;
                const T hyk = v ? hy[v - 1] : hyk0;
                const T hxk = v ? hx[v - 1] : hxk0;
                // the reference's zero differences at index 0: only the face's
                // own axis can reach it (the others start at P or P+1)
                DH<T> d;
                d.zy = (AX != 1 || j > 0) ? (hz[v] - hzj[v]) : T(0);
                d.yz = (AX != 2 || k > 0) ? (hy[v] - hyk) : T(0);
                d.xz = (AX != 2 || k > 0) ? (hx[v] - hxk) : T(0);
                d.zx = (AX != 0 || p > 0) ? (hz[v] - hzc[v]) : T(0);
                d.yx = (AX != 0 || p > 0) ? (hy[v] - hyc[v]) : T(0);
                d.xy = (AX != 1 || j > 0) ? (hx[v] - hxj[v]) : T(0);
                if ((AX == 0 && !ps) || (AX == 2 && rim_group && v == 0)) {
                    e_interior<T, LOSSY>(d, a.inv_dl, cax[v], cay[v], caz[v], cex[v], cey[v],
                                         cez[v], ex[v], ey[v], ez[v]);
                } else if (AX == 0) {
                    const T p_ey_x = bx * pa[v] + cx * d.zx;
                    const T p_ez_x = bx * pb[v] + cx * d.yx;
                    pa[v] = p_ey_x;
                    pb[v] = p_ez_x;
                    e_combine<T, LOSSY>(d, ikx, iky, ikz[v], T(0), T(0), p_ey_x, T(0), p_ez_x,
                                        T(0), cax[v], cay[v], caz[v], cex[v], cey[v], cez[v],
                                        ex[v], ey[v], ez[v]);
                } else if (AX == 1) {
                    const T p_ex_y = by * pa[v] + cy * d.zy;
                    const T p_ez_y = by * pb[v] + cy * d.xy;
                    pa[v] = p_ex_y;
                    pb[v] = p_ez_y;
                    e_combine<T, LOSSY>(d, ikx, iky, ikz[v], p_ex_y, T(0), T(0), T(0), T(0),
                                        p_ez_y, cax[v], cay[v], caz[v], cex[v], cey[v], cez[v],
                                        ex[v], ey[v], ez[v]);
                } else {
                    const T p_ex_z = bz[v] * pa[v] + cz[v] * d.yz;
                    const T p_ey_z = bz[v] * pb[v] + cz[v] * d.xz;
                    pa[v] = p_ex_z;
                    pb[v] = p_ey_z;
                    e_combine<T, LOSSY>(d, ikx, iky, ikz[v], T(0), p_ex_z, T(0), p_ey_z, T(0),
                                        T(0), cax[v], cay[v], caz[v], cex[v], cey[v], cez[v],
                                        ex[v], ey[v], ez[v]);
                }
            }
            const int64_t gi = (int64_t)p * sx + (int64_t)j * nz + kb;
            int64_t si = 0;
            if (AX == 0) si = ((int64_t)pml_layer(p, nx, npml) * ny + j) * nz + kb;
            if (AX == 1) si = ((int64_t)p * (2 * npml) + pml_layer(j, ny, npml)) * nz + kb;
            if (AX == 2) si = ((int64_t)p * ny + j) * (2 * npml) + pml_layer(kb, nz, npml);
            if (allv) {
                st_vec<T, V>(a.E_next[0] + gi, ex);
                st_vec<T, V>(a.E_next[1] + gi, ey);
                st_vec<T, V>(a.E_next[2] + gi, ez);
                if (ps) {
                    st_vec<T, V>(qa + si, pa);
                    st_vec<T, V>(qb + si, pb);
                }
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v)
                    if (kv[v]) {
                        a.E_next[0][gi + v] = ex[v];
                        a.E_next[1][gi + v] = ey[v];
                        a.E_next[2][gi + v] = ez[v];
                        if (ps && !rim_group) {
                            qa[si + v] = pa[v];
                            qb[si + v] = pb[v];
                        }
                    }
            }
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
            hyc[v] = hy[v];
            hzc[v] = hz[v];
        }
        __syncthreads();  // stage s is free
        if (tid == 0 && p + NSTAGE < i1) issue(p + NSTAGE);
    }
    if (!ok) {
        // drain: every copy issued must land before the CTA exits; only the
        // last NSTAGE issued planes can still be in flight
        __syncthreads();
        if (tid == 0) {
            const int from = max(pfirst, last_issued - NSTAGE + 1);
            for (int p = from; p <= last_issued; ++p) {
                const int s = (p - pfirst) % NSTAGE;
                const uint32_t par = ((p - pfirst) / NSTAGE) & 1;
                for (unsigned it = 0; it < FACE_DRAIN_LIMIT; ++it)
                    if (mbar_try_wait(&bar[s], par)) break;
            }
        }
        __syncthreads();
    }
}

// One launch for the six face regions: CTAs [f[a].first, f[a].first +
// f[a].ctas) march face a (AXS < 0), or one launch per face (AXS = a, CTAs
// from 0).  NSTAGE 4: two CTAs per SM; 3: three.
template <typename T, bool LOSSY, int NSTAGE, int AXS>
__global__ void __launch_bounds__(FACE_THREADS, NSTAGE == 3 ? 3 : 2)
    k_face_E(const __grid_constant__ FaceMaps maps, const YeeArgs<T> a,
             const __grid_constant__ FaceSet fs, const __grid_constant__ SourceList src) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const int b = blockIdx.x;
    if (AXS >= 0)
        face_march<T, LOSSY, NSTAGE, (AXS < 0 ? 0 : AXS)>(maps, a, fs, src, smem, b);
    else if (b - fs.f[0].first >= 0 && b - fs.f[0].first < fs.f[0].ctas)
        face_march<T, LOSSY, NSTAGE, 0>(maps, a, fs, src, smem, b - fs.f[0].first);
    else if (b - fs.f[1].first >= 0 && b - fs.f[1].first < fs.f[1].ctas)
        face_march<T, LOSSY, NSTAGE, 1>(maps, a, fs, src, smem, b - fs.f[1].first);
    else
        face_march<T, LOSSY, NSTAGE, 2>(maps, a, fs, src, smem, b - fs.f[2].first);
}

// Tuning knobs: FDTD_B200_FACE_NSTAGE=3 (three 3-stage CTAs per SM instead of
// two 4-stage ones), FDTD_B200_FACE_SPLIT=1 (one launch per face).
int face_nstage() {
    static const int v = [] {
        const char *e = getenv("FDTD_B200_FACE_NSTAGE");
        return (e && atoi(e) == 3) ? 3 : FACE_NSTAGE;
    }();
    return v;
}
bool face_split() {
    static const bool v = [] {
        const char *e = getenv("FDTD_B200_FACE_SPLIT");
        return e && atoi(e) == 1;
    }();
    return v;
}

template <typename T, bool LOSSY, int NSTAGE, int AXS>
cudaError_t launch_face_kernel(const FaceMaps &maps, const YeeArgs<T> &a, const FaceSet &fs,
                               const SourceList &src, int ctas, size_t smem, cudaStream_t st) {
    if (ctas <= 0) return cudaSuccess;
    cudaError_t e =
        ensure_max_dynamic_smem((const void *)k_face_E<T, LOSSY, NSTAGE, AXS>, (int)smem);
    if (e != cudaSuccess) return e;
    k_face_E<T, LOSSY, NSTAGE, AXS><<<ctas, FACE_THREADS, smem, st>>>(maps, a, fs, src);
    count_launches(1);
    return cudaGetLastError();
}

template <typename T, bool LOSSY, int NSTAGE>
cudaError_t launch_faces(const FaceMaps &maps, const YeeArgs<T> &a, const FaceSet &fs,
                         const SourceList &src, size_t smem, cudaStream_t st) {
    if (!face_split()) {
        const int all = fs.f[0].ctas + fs.f[1].ctas + fs.f[2].ctas;
        return launch_face_kernel<T, LOSSY, NSTAGE, -1>(maps, a, fs, src, all, smem, st);
    }
    cudaError_t e =
        launch_face_kernel<T, LOSSY, NSTAGE, 0>(maps, a, fs, src, fs.f[0].ctas, smem, st);
    if (e == cudaSuccess)
        e = launch_face_kernel<T, LOSSY, NSTAGE, 1>(maps, a, fs, src, fs.f[1].ctas, smem, st);
    if (e == cudaSuccess)
        e = launch_face_kernel<T, LOSSY, NSTAGE, 2>(maps, a, fs, src, fs.f[2].ctas, smem, st);
    return e;
}

template <typename T>
bool build_face_maps(const YeeArgs<T> &a, FaceMaps &m) {
    using L0 = FaceTile<T, 0>;
    using L2 = FaceTile<T, 2>;
    const int elem = (int)sizeof(T), nx = a.nx, ny = a.ny, nz = a.nz, p2 = 2 * a.npml;
    // the maps of this buffer set, built once
    static KeyedCache<FaceMaps, 20> cache;
    uint64_t key[20];
    for (int c = 0; c < 3; ++c) {
        key[c] = (uint64_t)(uintptr_t)a.E[c];
        key[3 + c] = (uint64_t)(uintptr_t)a.H_next[c];
        key[6 + c] = (uint64_t)(uintptr_t)a.ce[c];
        key[9 + c] = a.lossy ? (uint64_t)(uintptr_t)a.ca[c] : 0;
    }
    key[12] = (uint64_t)(uintptr_t)a.psi_e[0];
    key[13] = (uint64_t)(uintptr_t)a.psi_e[1];
    key[14] = (uint64_t)(uintptr_t)a.psi_e[2];
    key[15] = (uint64_t)(uintptr_t)a.psi_e[3];
    key[16] = (uint64_t)(uintptr_t)a.psi_e[4];
    key[17] = (uint64_t)(uintptr_t)a.psi_e[5];
    key[18] = ((uint64_t)nx << 40) ^ ((uint64_t)ny << 20) ^ (uint64_t)nz;
    key[19] = ((uint64_t)a.npml << 1) | (uint64_t)(a.lossy != 0);
    if (cache.get(key, m)) return true;
    memset(&m, 0, sizeof(m));
    const int hw[2] = {L0::HW, L2::HW}, hh[2] = {L0::HH, L2::HH};
    const int tk[2] = {L0::TK, L2::TK}, tj[2] = {L0::TJ, L2::TJ};
    // the z-face rows are 64-96 byte runs that no neighbouring tile shares:
    // no L2 promotion, so only their own sectors are fetched
    const int promo[2] = {256, 0};
    for (int sh = 0; sh < 2; ++sh)
        for (int c = 0; c < 3; ++c) {
            if (!make_tensor_map(&m.H[sh][c], a.H_next[c], nx, ny, nz, elem, hw[sh], hh[sh],
                                 promo[sh]) ||
                !make_tensor_map(&m.E[sh][c], a.E[c], nx, ny, nz, elem, tk[sh], tj[sh],
                                 promo[sh]) ||
                !make_tensor_map(&m.C[sh][c], a.ce[c], nx, ny, nz, elem, tk[sh], tj[sh],
                                 promo[sh]))
                return false;
            if (a.lossy && !make_tensor_map(&m.A[sh][c], a.ca[c], nx, ny, nz, elem, tk[sh],
                                            tj[sh], promo[sh]))
                return false;
        }
    // ψ stripes: x (2P, ny, nz), y (nx, 2P, nz), z (nx, ny, 2P)
    const bool ok =
        make_tensor_map(&m.P[0][0], a.psi_e[2], p2, ny, nz, elem, L0::TK, L0::TJ) &&
        make_tensor_map(&m.P[0][1], a.psi_e[4], p2, ny, nz, elem, L0::TK, L0::TJ) &&
        make_tensor_map(&m.P[1][0], a.psi_e[0], nx, p2, nz, elem, L0::TK, L0::TJ) &&
        make_tensor_map(&m.P[1][1], a.psi_e[5], nx, p2, nz, elem, L0::TK, L0::TJ) &&
        make_tensor_map(&m.P[2][0], a.psi_e[1], nx, ny, p2, elem, L2::TK, L2::TJ, 0) &&
        make_tensor_map(&m.P[2][1], a.psi_e[3], nx, ny, p2, elem, L2::TK, L2::TJ, 0);
    if (ok) cache.put(key, m);
    return ok;
}

void set_region(FaceBox &f, int r, const int lo[3], const int hi[3]) {
    for (int d = 0; d < 3; ++d) {
        f.lo[r][d] = lo[d];
        f.hi[r][d] = hi[d];
    }
}

int ceil_div(int a, int b) { return (a + b - 1) / b; }

// Chunks of about 16 planes along i.
void set_chunks(FaceBox &f, int nplanes) {
    f.nchunk = nplanes > 0 ? ceil_div(nplanes, 16) : 1;
    f.chunk = nplanes > 0 ? ceil_div(nplanes, f.nchunk) : 1;
}

// The face marches pay off only for a large shell: measured per step (FP32,
// one plane DFT, interleaved runs) they were slower than the per-cell kernel at
// 160x160x96 (86.2 against 73.7 us), 256^3 (312.6 / 311.3 us at npml 16) and
// 384^3 (859 / 851 us), and faster at 512^3 (1.854 / 1.877 ms, 24.3 M shell E
// cells); FP64 at 384^3 was slower too (1578.6 against 1562.2 us).
// FDTD_B200_FACE_E (read at every step) forces them on ("1", whenever the grid
// qualifies) or off ("0"); unset, they take shells of at least FACE_MIN_CELLS
// E cells.
constexpr int64_t FACE_MIN_CELLS = 20000000;

int face_mode() {
    const char *e = getenv("FDTD_B200_FACE_E");
    if (!e || !*e) return -1;
    return atoi(e) != 0 ? 1 : 0;
}

}  // namespace

// The six CPML face regions and the box list of the remaining shell E cells
// (P = npml, I = [P+1, N-P)): the x edges of the planes [0, P] and [N-P, N)
// (j or k in a CPML slab), the four y-z corner blocks of the I planes and the
// rim row j = P of the I planes.
static void face_partition(int nx, int ny, int nz, int P, int out_lo[6][3], int out_hi[6][3],
                           BoxPlan &rest) {
    const int reg[6][6] = {
        {0, P + 1, P, ny - P, P, nz - P},          {nx - P, nx, P, ny - P, P, nz - P},
        {P + 1, nx - P, 0, P, P, nz - P},          {P + 1, nx - P, ny - P, ny, P, nz - P},
        {P + 1, nx - P, P + 1, ny - P, 0, P + 1},  {P + 1, nx - P, P + 1, ny - P, nz - P, nz}};
    for (int q = 0; q < 6; ++q)
        for (int d = 0; d < 3; ++d) {
            out_lo[q][d] = reg[q][2 * d];
            out_hi[q][d] = reg[q][2 * d + 1];
        }
    memset(&rest, 0, sizeof(rest));
    const int xr[2][2] = {{0, P + 1}, {nx - P, nx}};
    for (int s = 0; s < 2; ++s) {
        const int a0 = xr[s][0], a1 = xr[s][1];
        plan_add(rest, a0, a1, 0, P, 0, nz);
        plan_add(rest, a0, a1, ny - P, ny, 0, nz);
        plan_add(rest, a0, a1, P, ny - P, 0, P);
        plan_add(rest, a0, a1, P, ny - P, nz - P, nz);
    }
    const int x0 = P + 1, x1 = nx - P;
    plan_add(rest, x0, x1, 0, P, 0, P);
    plan_add(rest, x0, x1, 0, P, nz - P, nz);
    plan_add(rest, x0, x1, ny - P, ny, 0, P);
    plan_add(rest, x0, x1, ny - P, ny, nz - P, nz);
    plan_add(rest, x0, x1, P, P + 1, 0, nz);
}

template <typename T>
bool face_path_ok(const YeeArgs<T> &a) {
    constexpr int V = 16 / (int)sizeof(T);
    const int P = a.npml;
    const int mode = face_mode();
    if (mode == 0 || P < V || P % V != 0 || a.nz % V != 0 || P + 1 > FACE_MAX_CHUNK)
        return false;
    if (a.xb.pml_lo != P || a.xb.pml_hi != P || a.ghost_lo != 0 || a.ghost_hi != 0) return false;
    if (a.nx - 2 * P < 2 || a.ny - 2 * P < 2 || a.nz - 2 * P < 2) return false;
    if (mode < 0) {
        const int64_t all = (int64_t)a.nx * a.ny * a.nz;
        const int64_t in = (int64_t)(a.nx - 2 * P - 1) * (a.ny - 2 * P - 1) * (a.nz - 2 * P - 1);
        if (all - in < FACE_MIN_CELLS) return false;
    }
    for (int c = 0; c < 3; ++c) {
        const void *ptrs[4] = {a.E[c], a.H_next[c], a.ce[c], a.E_next[c]};
        for (const void *q : ptrs)
            if (reinterpret_cast<uintptr_t>(q) % 16 != 0) return false;
        if (a.lossy && reinterpret_cast<uintptr_t>(a.ca[c]) % 16 != 0) return false;
    }
    for (int q = 0; q < 6; ++q)
        if (reinterpret_cast<uintptr_t>(a.psi_e[q]) % 16 != 0) return false;
    return true;
}

template <typename T>
cudaError_t launch_shell_E_faces(const YeeArgs<T> &a, const SourceList &src, cudaStream_t st,
                                 SideStream *side) {
    using L0 = FaceTile<T, 0>;
    using L2 = FaceTile<T, 2>;
    FaceMaps maps;
    // nothing launched yet: the caller takes the per-cell shell E instead
    if (!build_face_maps<T>(a, maps)) return cudaErrorNotSupported;
    int lo[6][3], hi[6][3];
    BoxPlan rest;
    face_partition(a.nx, a.ny, a.nz, a.npml, lo, hi, rest);
    FaceSet fs;
    memset(&fs, 0, sizeof(fs));
    for (int ax = 0; ax < 3; ++ax) {
        FaceBox &f = fs.f[ax];
        for (int r = 0; r < 2; ++r) set_region(f, r, lo[2 * ax + r], hi[2 * ax + r]);
        const int tk = ax == 2 ? L2::TK : L0::TK, tj = ax == 2 ? L2::TJ : L0::TJ;
        // both regions of a face have the same j extent
        f.ntj = ceil_div(f.hi[0][1] - f.lo[0][1], tj);
        for (int r = 0; r < 2; ++r) f.ntk[r] = ceil_div(f.hi[r][2] - f.lo[r][2], tk);
        if (ax == 0) {
            f.nchunk = 1;
            f.chunk = a.npml + 1;
        } else {
            set_chunks(f, f.hi[0][0] - f.lo[0][0]);
        }
        f.ctas = f.ntj * (f.ntk[0] + f.ntk[1]) * f.nchunk;
    }
    // launch order x, y, z (measured at 512³: the shell E phase took 0.388 ms
    // against 0.398 ms with the z faces first and 0.411 ms for the per-cell
    // kernel alone)
    fs.f[0].first = 0;
    fs.f[1].first = fs.f[0].ctas;
    fs.f[2].first = fs.f[1].first + fs.f[1].ctas;
    const bool lossy = a.lossy != 0;
    fs.stage_bytes = L0::stage_bytes(lossy) > L2::stage_bytes(lossy) ? L0::stage_bytes(lossy)
                                                                      : L2::stage_bytes(lossy);
    fs.wait_polls = interior_wait_polls();
    const int nstage = face_nstage();
    fs.bar_off = nstage * fs.stage_bytes;
    const size_t smem = fs.bar_off + 64 + 3 * FACE_MAX_CHUNK * sizeof(T) + 128;

    // the remaining cells on the side stream, concurrently (plane DFTs are
    // accumulated after both)
    PlaneList no_planes;
    memset(&no_planes, 0, sizeof(no_planes));
    cudaError_t e = cudaEventRecord(side->fork, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(side->s, side->fork, 0);
    if (e == cudaSuccess) e = launch_shell_E_boxes<T>(a, rest, src, no_planes, side->s);
    if (e != cudaSuccess) return e;
    if (lossy)
        e = nstage == 3 ? launch_faces<T, true, 3>(maps, a, fs, src, smem, st)
                        : launch_faces<T, true, FACE_NSTAGE>(maps, a, fs, src, smem, st);
    else
        e = nstage == 3 ? launch_faces<T, false, 3>(maps, a, fs, src, smem, st)
                        : launch_faces<T, false, FACE_NSTAGE>(maps, a, fs, src, smem, st);
    cudaError_t e2 = cudaEventRecord(side->join, side->s);
    if (e == cudaSuccess) e = e2;
    e2 = cudaStreamWaitEvent(st, side->join, 0);
    if (e == cudaSuccess) e = e2;
    return e;
}

template bool face_path_ok<float>(const YeeArgs<float> &);
template bool face_path_ok<double>(const YeeArgs<double> &);
template cudaError_t launch_shell_E_faces<float>(const YeeArgs<float> &, const SourceList &,
                                                 cudaStream_t, SideStream *);
template cudaError_t launch_shell_E_faces<double>(const YeeArgs<double> &, const SourceList &,
                                                  cudaStream_t, SideStream *);

int read_face_error(int reset) {
    int v = 0;
    cudaMemcpyFromSymbol(&v, g_face_error, sizeof(int));
    if (reset) {
        int z = 0;
        cudaMemcpyToSymbol(g_face_error, &z, sizeof(int));
    }
    return v;
}

}  // namespace fdtd
