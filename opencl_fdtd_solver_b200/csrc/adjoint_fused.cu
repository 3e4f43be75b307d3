// Fused reverse (adjoint) step for sm_100a: one pass over HBM for the interior.
//
// The transposed Yee step (adjoint.cu) has the shape of the forward step: H̄ is
// advanced from forward differences of Ē-side values, then Ē from backward
// differences of the new H̄.  In the CPML-free interior (κ = 1, no P terms) one
// reverse step of a cell is, with ik = 1/dl, u = (ce·ik)·Ē and v = (dtm·ik)·H̄',
//   H̄x' = H̄x + ((u_y − u_y[k+1]) + ((−u_z) − (−u_z[j+1])))
//   H̄y' = H̄y + (((−u_x) − (−u_x[k+1])) + (u_z − u_z[i+1]))
//   H̄z' = H̄z + ((u_x − u_x[j+1]) + ((−u_y) − (−u_y[i+1])))
//   Ēx' = Ēx + (((−v_y[k−1]) − (−v_y)) + (v_z[j−1] − v_z))
//   Ēy' = Ēy + ((v_x[k−1] − v_x) + ((−v_z[i−1]) − (−v_z)))
//   Ēz' = Ēz + (((−v_x[j−1]) − (−v_x)) + (v_y[i−1] − v_y))
// which are the fast-path expressions of adj_h_cell / adj_e_cell operand for
// operand, so with --fmad=false every cell equals the per-cell kernels bit for
// bit.  The gradient Σ Ē·(E^{n+1} − E^n) of the gradient-box cells the march
// updates is accumulated by extra threads of the shell-H̄ launch (its dependent
// global reads stalled the march when done inside it: 98 against 29 µs at
// 160 x 160 x 96), from Ē before the step, with the operations of adj_h_cell.
//
// Schedule of one fused reverse step (reads Ē, H̄, P; writes Ē', H̄', P'), three
// launches on the caller's stream: k_adj_shell_H on the cells outside HB =
// [npml, N-npml-1)^3 (extra threads accumulate the gradient of the gradient-box
// cells inside HB), k_adj_interior (H̄' on HB, Ē' on EB = [npml+1, N-npml-1)^3),
// k_adj_shell_E on the cells outside EB; the objective's seed is added to Ē' in
// the last two, in the order adj_e_cell adds it.
//
// Interior kernel: each CTA owns a (TJ x TK) tile of (j, k) and marches along i
// over a chunk of planes.  Plane p arrives by TMA (cp.async.bulk.tensor 3-D
// tiled maps, no multicast) in an NSTAGE-deep ring completed by mbarrier
// transaction counts: Ē(p) and ce(p) over rows j0-1 .. j0+TJ and columns
// k0-V .. k0+TK+V-1, H̄(p) over rows j0-1 .. j0+TJ-1 and columns k0-V ..
// k0+TK-1.  128 threads update V consecutive k cells each with 16-byte
// shared-memory vectors; a fifth warp recomputes H̄' of the j0-1 row and the
// k0-1 column.  Ē' uses H̄'(p) from shared memory and H̄'(p-1) carried in
// registers.  HBM traffic per interior cell: Ē, H̄, ce read once, Ē', H̄'
// written once (60 B FP32).  Every mbarrier wait is bounded (the interior wait
// budget); on timeout the kernel raises bit 2 of the device error flag, waits
// for the copies it issued and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "adjoint.cuh"
#include "launch_count.cuh"
#include "tma.cuh"

namespace fdtd {

int interior_chunks(int tiles, int nplanes, int sms);

namespace {

__device__ int g_adj_error = 0;

constexpr int A_NSTAGE = 4;
constexpr int A_NCELL = 128;              // 16 vector groups x 8 rows
constexpr int A_NTHREADS = A_NCELL + 32;  // + one halo warp
constexpr unsigned A_DRAIN = (1u << 24) / 16;

// G vector groups of V cells per row: 16 (TK x TJ = 64 x 8 FP32) or 8 (32 x
// 16), whichever pads the box's k extent less (same halo ratio and bytes).
template <typename T, int GG>
struct ATile {
    static constexpr int V = 16 / (int)sizeof(T);
    static constexpr int G = GG;
    static constexpr int TK = G * V;
    static constexpr int TJ = A_NCELL / G;
    static constexpr int EW = TK + 2 * V, EH = TJ + 2;
    static constexpr int HW = TK + V, HH = TJ + 1;
    __host__ __device__ static constexpr int pad128(int b) { return (b + 127) / 128 * 128; }
    static constexpr int EB = pad128(EW * EH * (int)sizeof(T));
    static constexpr int HB = pad128(HW * HH * (int)sizeof(T));
    static constexpr int STAGE = 6 * EB + 3 * HB;  // Ē, ce (E box) and H̄
    static constexpr uint32_t TX_FULL = 3u * (2 * EW * EH + HW * HH) * sizeof(T);
    static constexpr uint32_t TX_E = 3u * 2 * EW * EH * sizeof(T);  // Ē and ce only
};

struct alignas(64) AdjMaps {
    CUtensorMap E[3];
    CUtensorMap C[3];
    CUtensorMap H[3];
};

struct AdjBox {
    int lo[3], hi[3];  // H̄ box HB = [lo, hi); Ē box EB = [lo+1, hi)
    int j0base, k0base, ntk, chunk;
    unsigned wait_polls;
    int new_off, bar_off;
};

template <typename T>
struct AdjMarch {
    int nx, ny, nz;
    T ik, wk;  // 1/dl and dtm/dl as the per-cell kernels round them
    T *Eo[3];
    T *Ho[3];
    AdjSeed sd;  // the objective's seed, added to Ē' of its patch cells
};

__device__ __forceinline__ bool adj_wait(uint64_t *bar, uint32_t parity, unsigned limit) {
    if (limit == 0) {
        if (mbar_test_wait(bar, parity)) return true;
    } else {
        for (unsigned it = 0; it < limit; ++it)
            if (mbar_try_wait(bar, parity)) return true;
    }
    atomicOr(&g_adj_error, 1);
    return false;
}

template <typename T, int NSTAGE, int GG>
__global__ void __launch_bounds__(A_NTHREADS, 2)
    k_adj_interior(const __grid_constant__ AdjMaps maps, const __grid_constant__ AdjMarch<T> m,
                   const __grid_constant__ AdjBox bx) {
    using L = ATile<T, GG>;
    constexpr int V = L::V, TK = L::TK, TJ = L::TJ, EW = L::EW, HW = L::HW;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + bx.bar_off);

    const int ny = m.ny, nz = m.nz;
    const int tile = blockIdx.x;
    const int k0 = bx.k0base + (tile % bx.ntk) * TK;
    const int j0 = bx.j0base + (tile / bx.ntk) * TJ;
    const int i0 = bx.lo[0] + blockIdx.y * bx.chunk;
    const int i1 = min(bx.hi[0], i0 + bx.chunk);
    const int pfirst = (i0 > bx.lo[0]) ? i0 - 1 : i0;  // pre-plane recomputes H̄'(i0-1)
    const int plast = i1;                               // Ē, ce only
    const int tid = threadIdx.x;
    const bool cell_thr = tid < A_NCELL;
    const int g = tid % L::G, r = tid / L::G;

    auto sE = [&](int s, int c) { return reinterpret_cast<T *>(smem + s * L::STAGE + c * L::EB); };
    auto sC = [&](int s, int c) {
        return reinterpret_cast<T *>(smem + s * L::STAGE + (3 + c) * L::EB);
    };
    auto sH = [&](int s, int c) {
        return reinterpret_cast<T *>(smem + s * L::STAGE + 6 * L::EB + c * L::HB);
    };
    auto sN = [&](int c) { return reinterpret_cast<T *>(smem + bx.new_off + c * L::HB); };
    if (tid == 0) {
        for (int s = 0; s < NSTAGE; ++s) mbar_init(&bar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();

    int last_issued = pfirst - 1;  // thread 0 only
    auto issue = [&](int p) {
        const int s = (p - pfirst) % NSTAGE;
        last_issued = p;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&bar[s], p < plast ? L::TX_FULL : L::TX_E);
        for (int c = 0; c < 3; ++c) {
            tma_load_3d(sE(s, c), &maps.E[c], &bar[s], k0 - V, j0 - 1, p);
            tma_load_3d(sC(s, c), &maps.C[c], &bar[s], k0 - V, j0 - 1, p);
            if (p < plast) tma_load_3d(sH(s, c), &maps.H[c], &bar[s], k0 - V, j0 - 1, p);
        }
    };
    if (tid == 0)
        for (int p = pfirst; p <= plast && p < pfirst + NSTAGE; ++p) issue(p);

    const T ik = m.ik, wk = m.wk;
    const int64_t sx = (int64_t)ny * nz;
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
    const int ho = (r + 1) * HW + V + V * g;  // own cells in the H box
    // the u of one E-box position: (ce·ik)·Ē
    auto uval = [&](const T *e, const T *c, int o) { return (c[o] * ik) * e[o]; };

    T hyc[V], hzc[V];  // H̄'(p-1) at own cells
#pragma unroll
    for (int v = 0; v < V; ++v) hyc[v] = hzc[v] = T(0);

    bool ok = true;
    for (int p = pfirst; p < plast; ++p) {
        const int s = (p - pfirst) % NSTAGE, s1 = (p + 1 - pfirst) % NSTAGE;
        const uint32_t par = ((p - pfirst) / NSTAGE) & 1, par1 = ((p + 1 - pfirst) / NSTAGE) & 1;
        const bool w = adj_wait(&bar[s], par, bx.wait_polls) && adj_wait(&bar[s1], par1, bx.wait_polls);
        if (!__syncthreads_and(w)) {
            ok = false;
            break;
        }
        const bool storeH = p >= i0;
        const bool doE = p >= i0 && p >= bx.lo[0] + 1;
        const T *E0x = sE(s, 0), *E0y = sE(s, 1), *E0z = sE(s, 2);
        const T *C0x = sC(s, 0), *C0y = sC(s, 1), *C0z = sC(s, 2);
        const T *E1y = sE(s1, 1), *E1z = sE(s1, 2), *C1y = sC(s1, 1), *C1z = sC(s1, 2);
        T ex0[V], ey0[V], ez0[V], hx[V], hy[V], hz[V];
        if (cell_thr) {
            T cx[V], cy[V], cz[V], ux[V], uy[V], uz[V];
            ld_vec<T, V>(E0x + eo, ex0);
            ld_vec<T, V>(E0y + eo, ey0);
            ld_vec<T, V>(E0z + eo, ez0);
            ld_vec<T, V>(C0x + eo, cx);
            ld_vec<T, V>(C0y + eo, cy);
            ld_vec<T, V>(C0z + eo, cz);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                ux[v] = (cx[v] * ik) * ex0[v];
                uy[v] = (cy[v] * ik) * ey0[v];
                uz[v] = (cz[v] * ik) * ez0[v];
            }
            ld_vec<T, V>(sH(s, 0) + ho, hx);
            ld_vec<T, V>(sH(s, 1) + ho, hy);
            ld_vec<T, V>(sH(s, 2) + ho, hz);
            // k+1 of the last cell: the next thread's first, or the halo column
            T uxn = __shfl_down_sync(0xffffffffu, ux[0], 1);
            T uyn = __shfl_down_sync(0xffffffffu, uy[0], 1);
            if (g == L::G - 1) {
                uxn = uval(E0x, C0x, eo + V);
                uyn = uval(E0y, C0y, eo + V);
            }
            // the j+1 row (x, z) and the i+1 plane (y, z) as 16-byte vectors
            T exj[V], ezj[V], cxj[V], czj[V], eyi[V], ezi[V], cyi[V], czi[V];
            ld_vec<T, V>(E0x + eo + EW, exj);
            ld_vec<T, V>(C0x + eo + EW, cxj);
            ld_vec<T, V>(E0z + eo + EW, ezj);
            ld_vec<T, V>(C0z + eo + EW, czj);
            ld_vec<T, V>(E1y + eo, eyi);
            ld_vec<T, V>(C1y + eo, cyi);
            ld_vec<T, V>(E1z + eo, ezi);
            ld_vec<T, V>(C1z + eo, czi);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const T uxk = (v < V - 1) ? ux[v + 1] : uxn;
                const T uyk = (v < V - 1) ? uy[v + 1] : uyn;
                const T uxj = (cxj[v] * ik) * exj[v], uzj = (czj[v] * ik) * ezj[v];
                const T uyi = (cyi[v] * ik) * eyi[v], uzi = (czi[v] * ik) * ezi[v];
                hx[v] = hx[v] + ((uy[v] - uyk) + ((-uz[v]) - (-uzj)));
                hy[v] = hy[v] + (((-ux[v]) - (-uxk)) + (uz[v] - uzi));
                hz[v] = hz[v] + ((ux[v] - uxj) + ((-uy[v]) - (-uyi)));
            }
            st_vec<T, V>(sN(0) + ho, hx);
            st_vec<T, V>(sN(1) + ho, hy);
            st_vec<T, V>(sN(2) + ho, hz);
            if (storeH && rowH) {
                const int64_t gi = (int64_t)p * sx + (int64_t)j * nz + kb;
                if (allH) {
                    st_vec<T, V>(m.Ho[0] + gi, hx);
                    st_vec<T, V>(m.Ho[1] + gi, hy);
                    st_vec<T, V>(m.Ho[2] + gi, hz);
                } else {
#pragma unroll
                    for (int v = 0; v < V; ++v)
                        if (kH[v]) {
                            m.Ho[0][gi + v] = hx[v];
                            m.Ho[1][gi + v] = hy[v];
                            m.Ho[2][gi + v] = hz[v];
                        }
                }
            }
        } else if (doE) {
            // halo warp: H̄' on row j0-1 (lanes 0..15) and column k0-1 (lanes 16..23)
            const int lane = tid - A_NCELL;
            if (lane < L::G) {
                if (j0 - 1 >= bx.lo[1]) {
                    const int e = V + V * lane, h = V + V * lane;
                    T qx[V], qy[V], qz[V];
                    ld_vec<T, V>(sH(s, 0) + h, qx);
                    ld_vec<T, V>(sH(s, 1) + h, qy);
                    ld_vec<T, V>(sH(s, 2) + h, qz);
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        const T ux = uval(E0x, C0x, e + v), uy = uval(E0y, C0y, e + v);
                        const T uz = uval(E0z, C0z, e + v);
                        const T uxk = uval(E0x, C0x, e + v + 1), uyk = uval(E0y, C0y, e + v + 1);
                        const T uxj = uval(E0x, C0x, e + EW + v), uzj = uval(E0z, C0z, e + EW + v);
                        const T uyi = uval(E1y, C1y, e + v), uzi = uval(E1z, C1z, e + v);
                        qx[v] = qx[v] + ((uy - uyk) + ((-uz) - (-uzj)));
                        qy[v] = qy[v] + (((-ux) - (-uxk)) + (uz - uzi));
                        qz[v] = qz[v] + ((ux - uxj) + ((-uy) - (-uyi)));
                    }
                    st_vec<T, V>(sN(0) + h, qx);
                    st_vec<T, V>(sN(1) + h, qy);
                    st_vec<T, V>(sN(2) + h, qz);
                }
            } else if (lane < L::G + TJ) {
                const int rr = lane - L::G;
                if (k0 - 1 >= bx.lo[2] && j0 + rr < ny) {
                    const int e = (rr + 1) * EW + V - 1, h = (rr + 1) * HW + V - 1;
                    const T ux = uval(E0x, C0x, e), uy = uval(E0y, C0y, e), uz = uval(E0z, C0z, e);
                    const T uxk = uval(E0x, C0x, e + 1), uyk = uval(E0y, C0y, e + 1);
                    const T uxj = uval(E0x, C0x, e + EW), uzj = uval(E0z, C0z, e + EW);
                    const T uyi = uval(E1y, C1y, e), uzi = uval(E1z, C1z, e);
                    sN(0)[h] = sH(s, 0)[h] + ((uy - uyk) + ((-uz) - (-uzj)));
                    sN(1)[h] = sH(s, 1)[h] + (((-ux) - (-uxk)) + (uz - uzi));
                    sN(2)[h] = sH(s, 2)[h] + ((ux - uxj) + ((-uy) - (-uyi)));
                }
            }
        }
        __syncthreads();

        T vyk0 = T(0), vxk0 = T(0);  // H̄'y, H̄'x at k-1 of the first cell
        if (doE && cell_thr) {
            vyk0 = __shfl_up_sync(0xffffffffu, hy[V - 1], 1);
            vxk0 = __shfl_up_sync(0xffffffffu, hx[V - 1], 1);
            if (g == 0) {
                vyk0 = sN(1)[ho - 1];
                vxk0 = sN(0)[ho - 1];
            }
        }
        if (doE && cell_thr && rowE) {
            T hzj[V], hxj[V];
            ld_vec<T, V>(sN(2) + ho - HW, hzj);
            ld_vec<T, V>(sN(0) + ho - HW, hxj);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const T hyk = v ? hy[v - 1] : vyk0;
                const T hxk = v ? hx[v - 1] : vxk0;
                const T a3 = -(wk * hy[v]), a3p = -(wk * hyk);
                const T a5 = wk * hz[v], a5p = wk * hzj[v];
                const T a1 = wk * hx[v], a1p = wk * hxk;
                const T a4 = -(wk * hz[v]), a4p = -(wk * hzc[v]);
                const T a0 = -(wk * hx[v]), a0p = -(wk * hxj[v]);
                const T a2 = wk * hy[v], a2p = wk * hyc[v];
                ex0[v] = ex0[v] + ((a3p - a3) + (a5p - a5));
                ey0[v] = ey0[v] + ((a1p - a1) + (a4p - a4));
                ez0[v] = ez0[v] + ((a0p - a0) + (a2p - a2));
                if (m.sd.active && kE[v]) add_seed<T>(m.sd, p, j, kb + v, ex0[v], ey0[v], ez0[v]);
            }
            const int64_t gi = (int64_t)p * sx + (int64_t)j * nz + kb;
            if (allE) {
                st_vec<T, V>(m.Eo[0] + gi, ex0);
                st_vec<T, V>(m.Eo[1] + gi, ey0);
                st_vec<T, V>(m.Eo[2] + gi, ez0);
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v)
                    if (kE[v]) {
                        m.Eo[0][gi + v] = ex0[v];
                        m.Eo[1][gi + v] = ey0[v];
                        m.Eo[2][gi + v] = ez0[v];
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
        __syncthreads();  // stage s and the new-H̄ plane are free
        if (tid == 0 && p + NSTAGE <= plast) issue(p + NSTAGE);
    }
    if (!ok) {
        // every copy issued lands before the CTA exits (only the last NSTAGE
        // issued planes can still be in flight)
        __syncthreads();
        if (tid == 0) {
            const int from = max(pfirst, last_issued - NSTAGE + 1);
            for (int p = from; p <= last_issued; ++p) {
                const int s = (p - pfirst) % NSTAGE;
                const uint32_t par = ((p - pfirst) / NSTAGE) & 1;
                for (unsigned it = 0; it < A_DRAIN; ++it)
                    if (mbar_try_wait(&bar[s], par)) break;
            }
        }
        __syncthreads();
    }
}

template <typename T, int GG>
bool adj_maps(const AdjArgs<T> &a, AdjMaps &maps) {
    using L = ATile<T, GG>;
    const int elem = (int)sizeof(T);
    memset(&maps, 0, sizeof(maps));
    for (int c = 0; c < 3; ++c)
        if (!make_tensor_map(&maps.E[c], a.E[c], a.nx, a.ny, a.nz, elem, L::EW, L::EH) ||
            !make_tensor_map(&maps.C[c], a.ce[c], a.nx, a.ny, a.nz, elem, L::EW, L::EH) ||
            !make_tensor_map(&maps.H[c], a.H[c], a.nx, a.ny, a.nz, elem, L::HW, L::HH))
            return false;
    return true;
}

template <typename T, int GG>
cudaError_t launch_adj_interior(const AdjArgs<T> &a, const AdjSeed &sd, const AdjOut<T> &out,
                                const AdjMaps &maps, const ShellBox &hb, cudaStream_t st) {
    using L = ATile<T, GG>;
    AdjBox bx;
    for (int d = 0; d < 3; ++d) {
        bx.lo[d] = hb.lo[d];
        bx.hi[d] = hb.hi[d];
    }
    bx.k0base = (hb.lo[2] / L::V) * L::V;  // 16-byte aligned TMA x coordinates
    bx.j0base = hb.lo[1];
    bx.ntk = (hb.hi[2] - bx.k0base + L::TK - 1) / L::TK;
    const int ntj = (hb.hi[1] - bx.j0base + L::TJ - 1) / L::TJ;
    const int tiles = bx.ntk * ntj;
    const int sms = device_sm_count();
    const int nplanes = hb.hi[0] - hb.lo[0];
    const int nchunk = interior_chunks(tiles, nplanes, sms);
    bx.chunk = (nplanes + nchunk - 1) / nchunk;
    bx.wait_polls = interior_wait_polls();
    bx.new_off = A_NSTAGE * L::STAGE;
    bx.bar_off = bx.new_off + 3 * L::HB;
    const size_t smem = bx.bar_off + 64 + 128;
    AdjMarch<T> m;
    m.nx = a.nx;
    m.ny = a.ny;
    m.nz = a.nz;
    m.ik = a.ik_int;
    m.wk = a.dtm * a.ik_int;
    for (int c = 0; c < 3; ++c) {
        m.Eo[c] = out.E[c];
        m.Ho[c] = out.H[c];
    }
    m.sd = sd;
    dim3 grid(tiles, (nplanes + bx.chunk - 1) / bx.chunk, 1);
    cudaError_t e =
        ensure_max_dynamic_smem((const void *)k_adj_interior<T, A_NSTAGE, GG>, (int)smem);
    if (e != cudaSuccess) return e;
    k_adj_interior<T, A_NSTAGE, GG><<<grid, A_NTHREADS, smem, st>>>(maps, m, bx);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace

template <typename T>
cudaError_t launch_adjoint_step_fused(const AdjArgs<T> &a, const AdjGrad<T> &gb,
                                      const AdjSeed &sd, const AdjOut<T> &out, cudaStream_t st) {
    const int elem = (int)sizeof(T);
    const int n[3] = {a.nx, a.ny, a.nz};
    // HB = [npml, N-npml-1)^3: cells whose H̄ update (cell and +1 neighbours) has
    // no P terms; EB = [npml+1, N-npml-1)^3 likewise for Ē (cell and -1)
    bool march = a.npml >= 1 && ((int64_t)a.nz * elem) % 16 == 0;
    for (int d = 0; d < 3; ++d) march = march && n[d] - 2 * a.npml - 1 >= 2;
    for (int c = 0; c < 3 && march; ++c) {
        const void *ptrs[5] = {a.E[c], a.H[c], a.ce[c], out.E[c], out.H[c]};
        for (const void *q : ptrs)
            if (reinterpret_cast<uintptr_t>(q) % 16 != 0) march = false;
    }
    int gsel = 16;
    {
        const int V = ATile<T, 16>::V, k0 = (a.npml / V) * V, ext = (n[2] - a.npml - 1) - k0;
        const int w16 = ATile<T, 16>::TK, w8 = ATile<T, 8>::TK;
        // 64 x 8 streams better (measured at 512³: 1.18 ms against 1.31 ms for the
        // 32 x 16 tile, which pads 480 cells to 480 instead of 512); the 32 x 16
        // tile is taken only where it saves a fifth of the padded k extent
        if (5 * ((ext + w16 - 1) / w16 * w16) > 6 * ((ext + w8 - 1) / w8 * w8)) gsel = 8;
    }
    AdjMaps maps;
    if (march && !(gsel == 8 ? adj_maps<T, 8>(a, maps) : adj_maps<T, 16>(a, maps))) march = false;
    if (!march) {
        // grid-wide per-cell kernels into the outputs, then the seed (the same
        // result as the in-place path)
        AdjSeed none = sd;
        none.active = 0;
        cudaError_t e = launch_adjoint_grid<T>(a, gb, none, out, st);
        if (e == cudaSuccess && sd.active)
            e = launch_adjoint_seed<T>(a.nx, a.ny, a.nz, out.E, sd, st);
        return e;
    }
    ShellBox hb, eb, all;
    for (int d = 0; d < 3; ++d) {
        hb.lo[d] = a.npml;
        hb.hi[d] = n[d] - a.npml - 1;
        eb.lo[d] = a.npml + 1;
        eb.hi[d] = n[d] - a.npml - 1;
        all.lo[d] = 0;
        all.hi[d] = n[d];
    }
    // three launches on the caller's stream: shell H̄ (whose extra threads also
    // accumulate the gradient of the march's cells), the march, shell Ē; the
    // seed is added in the Ē epilogues of the last two.  (On a side stream
    // beside the march the shell kernels were starved; as separate launches the
    // gradient and seed kernels added gaps between short dependent kernels.)
    ShellBox gx;
    for (int d = 0; d < 3; ++d) {
        gx.lo[d] = gb.lo[d] > hb.lo[d] ? gb.lo[d] : hb.lo[d];
        gx.hi[d] = gb.hi[d] < hb.hi[d] ? gb.hi[d] : hb.hi[d];
        if (!gb.active || gx.hi[d] < gx.lo[d]) gx.hi[d] = gx.lo[d];
    }
    cudaError_t e = launch_adjoint_shell_H<T>(a, gb, out, all, hb, gx, st);
    if (e == cudaSuccess)
        e = gsel == 8 ? launch_adj_interior<T, 8>(a, sd, out, maps, hb, st)
                      : launch_adj_interior<T, 16>(a, sd, out, maps, hb, st);
    if (e == cudaSuccess) e = launch_adjoint_shell_E<T>(a, sd, out, all, eb, st);
    return e;
}

template cudaError_t launch_adjoint_step_fused<float>(const AdjArgs<float> &,
                                                      const AdjGrad<float> &, const AdjSeed &,
                                                      const AdjOut<float> &, cudaStream_t);
template cudaError_t launch_adjoint_step_fused<double>(const AdjArgs<double> &,
                                                       const AdjGrad<double> &, const AdjSeed &,
                                                       const AdjOut<double> &, cudaStream_t);

int read_adjoint_error(int reset) {
    int v = 0;
    cudaMemcpyFromSymbol(&v, g_adj_error, sizeof(int));
    if (reset) {
        int z = 0;
        cudaMemcpyToSymbol(g_adj_error, &z, sizeof(int));
    }
    return v;
}

}  // namespace fdtd
