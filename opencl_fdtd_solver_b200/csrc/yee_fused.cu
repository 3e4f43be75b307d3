// Fused single-pass Yee step for sm_100a: H^{n-1/2} -> H^{n+1/2}, sheet
// injections, E^n -> E^{n+1} and plane DFTs in one sweep over HBM.
//
// Schedule.  Each CTA owns a (TJ x TK) tile of (j, k) and marches along i over
// a chunk of planes [i0, i1).  Plane p of the input fields is brought into
// shared memory by TMA (cp.async.bulk.tensor, 3-D tiled maps, no multicast):
//   E^n(p)       rows j0-1 .. j0+TJ, cols k0-HP .. k0+TK+HP-1  (1-cell halo;
//                the k extent is widened to 16-byte boundaries)
//   H^{n-1/2}(p) rows j0-1 .. j0+TJ-1, cols k0-HP .. k0+TK-1
//   ce(p) [ca(p)] the tile only
// through an NSTAGE-deep ring of stages, each completed by one mbarrier with a
// transaction-byte count.  Per plane the CTA computes H^{n+1/2}(p) on the tile
// plus the j0-1 row and k0-1 column that the E stencil needs (recomputed from
// the same inputs, so no inter-CTA exchange), then E^{n+1}(p) on the tile from
// H^{n+1/2}(p) (shared memory) and H^{n+1/2}(p-1) (carried in registers).
// Outputs go to separate buffers (E_next, H_next, psi_h_next), so no CTA ever
// reads a value another CTA has already overwritten; psi_e is per-cell and
// updated in place.  A chunk starting at i0 > 0 first recomputes
// H^{n+1/2}(i0-1) for its tile (no stores).
//
// HBM traffic per cell: E, H, ce read once and E, H written once (60 B in FP32
// lossless), plus the CPML stripes and the plane-DFT accumulators.
//
// Arithmetic: the per-cell expressions are those of yee_cell.cuh, compiled
// with --fmad=false, so results equal the split kernels and the CPU oracle bit
// for bit.
//
// Every mbarrier wait is bounded; on timeout the kernel raises a device error
// flag, drains its outstanding copies (bounded again) and returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <unordered_map>

#include "yee_launch.cuh"

namespace fdtd {

__device__ int g_fused_error = 0;

constexpr int NSTAGE = 4;
constexpr int NTHREADS = 256;
constexpr unsigned WAIT_LIMIT = 1u << 24;

struct alignas(64) FusedMaps {
    CUtensorMap E[3];
    CUtensorMap H[3];
    CUtensorMap C[3];
    CUtensorMap A[3];
};

template <typename T>
struct FusedTile {
    static constexpr int TK = (sizeof(T) == 4) ? 64 : 32;  // 256-byte rows
    static constexpr int TJ = 8;
    static constexpr int HP = 16 / (int)sizeof(T);         // 16-byte k alignment pad
    static constexpr int NTY = NTHREADS / TK;
    static constexpr int RPT = TJ / NTY;                    // rows per thread
    static constexpr int EW = TK + 2 * HP, EH = TJ + 2;
    static constexpr int HW = TK + HP, HH = TJ + 1;
    static constexpr int NW = TK + 1, NH = TJ + 1;          // new-H plane incl. halo
    __host__ __device__ static constexpr int pad128(int b) { return (b + 127) / 128 * 128; }
    static constexpr int EB = pad128(EW * EH * (int)sizeof(T));
    static constexpr int HB = pad128(HW * HH * (int)sizeof(T));
    static constexpr int CB = pad128(TK * TJ * (int)sizeof(T));
    __host__ __device__ static constexpr int stage_bytes(bool lossy) {
        return 3 * EB + 3 * HB + 3 * CB * (lossy ? 2 : 1);
    }
    static constexpr int NB = pad128(3 * NW * NH * (int)sizeof(T));
    __host__ __device__ static constexpr int smem_bytes(bool lossy) {
        return NSTAGE * stage_bytes(lossy) + NB + 256;
    }
    // bytes a full stage (E, H, ce[, ca]) and an E-only stage deliver
    __host__ __device__ static constexpr uint32_t tx_full(bool lossy) {
        return 3u * (EW * EH + HW * HH + TK * TJ * (lossy ? 2 : 1)) * sizeof(T);
    }
    __host__ __device__ static constexpr uint32_t tx_eonly() { return 3u * EW * EH * sizeof(T); }
};

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false (and the device error flag set) if the phase did not
// complete within WAIT_LIMIT polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    for (unsigned it = 0; it < WAIT_LIMIT; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    atomicOr(&g_fused_error, 1);
    return false;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int c0, int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

// ---------------------------------------------------------------- the kernel
template <typename T, bool LOSSY>
__global__ void __launch_bounds__(NTHREADS, 2)
    k_step_fused(const __grid_constant__ FusedMaps maps, const YeeArgs<T> a,
                 const SourceList src, const PlaneList planes, int ntk, int chunk) {
    using L = FusedTile<T>;
    constexpr int TK = L::TK, TJ = L::TJ, HP = L::HP, NTY = L::NTY, RPT = L::RPT;
    constexpr int EW = L::EW, EH = L::EH, HW = L::HW, NW = L::NW;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    constexpr int SB = L::stage_bytes(LOSSY);
    T *sNew = reinterpret_cast<T *>(smem + NSTAGE * SB);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + NSTAGE * SB + L::NB);

    const int nx = a.nx, ny = a.ny, nz = a.nz, npml = a.npml;
    const int tile = blockIdx.x;
    const int k0 = (tile % ntk) * TK;
    const int j0 = (tile / ntk) * TJ;
    const int i0 = blockIdx.y * chunk;
    const int i1 = min(nx, i0 + chunk);
    const int pfirst = (i0 > 0) ? i0 - 1 : 0;  // first plane whose H^{n+1/2} is computed
    const int plast = i1;                      // last plane loaded (E only when == i1)
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * TK + tx;

    auto stage_ptr = [&](int s) { return smem + s * SB; };
    auto sE = [&](int s, int c) { return reinterpret_cast<T *>(stage_ptr(s) + c * L::EB); };
    auto sH = [&](int s, int c) {
        return reinterpret_cast<T *>(stage_ptr(s) + 3 * L::EB + c * L::HB);
    };
    auto sC = [&](int s, int c) {
        return reinterpret_cast<T *>(stage_ptr(s) + 3 * L::EB + 3 * L::HB + c * L::CB);
    };
    auto sA = [&](int s, int c) {
        return reinterpret_cast<T *>(stage_ptr(s) + 3 * L::EB + 3 * L::HB + (3 + c) * L::CB);
    };

    if (tid == 0) {
        for (int s = 0; s < NSTAGE; ++s) mbar_init(&bar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();

    // producer: issue the loads of plane p into its stage
    auto issue = [&](int p) {
        const int s = (p - pfirst) % NSTAGE;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (p < plast) {
            mbar_expect_tx(&bar[s], L::tx_full(LOSSY));
            for (int c = 0; c < 3; ++c) {
                tma_load_3d(sE(s, c), &maps.E[c], &bar[s], k0 - HP, j0 - 1, p);
                tma_load_3d(sH(s, c), &maps.H[c], &bar[s], k0 - HP, j0 - 1, p);
                tma_load_3d(sC(s, c), &maps.C[c], &bar[s], k0, j0, p);
                if (LOSSY) tma_load_3d(sA(s, c), &maps.A[c], &bar[s], k0, j0, p);
            }
        } else {
            mbar_expect_tx(&bar[s], L::tx_eonly());
            for (int c = 0; c < 3; ++c) tma_load_3d(sE(s, c), &maps.E[c], &bar[s], k0 - HP, j0 - 1, p);
        }
    };
    if (tid == 0)
        for (int p = pfirst; p <= plast && p < pfirst + NSTAGE; ++p) issue(p);

    const T dtm = a.dtm, dtm_dl = a.dtm_dl, inv_dl = a.inv_dl;
    const int64_t sx = (int64_t)ny * nz, sy = nz;

    T carry_hy[RPT], carry_hz[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) carry_hy[r] = carry_hz[r] = T(0);

    bool ok = true;
    for (int p = pfirst; p < plast; ++p) {
        const int s = (p - pfirst) % NSTAGE, s1 = (p + 1 - pfirst) % NSTAGE;
        const uint32_t par = ((p - pfirst) / NSTAGE) & 1, par1 = ((p + 1 - pfirst) / NSTAGE) & 1;
        const bool w = mbar_wait(&bar[s], par) && mbar_wait(&bar[s1], par1);
        if (!__syncthreads_and(w)) {  // CTA-uniform exit on a timed-out copy
            ok = false;
            break;
        }
        const bool real_plane = (p >= i0);
        const T *E0[3] = {sE(s, 0), sE(s, 1), sE(s, 2)};
        const T *E1[3] = {sE(s1, 0), sE(s1, 1), sE(s1, 2)};
        const T *H0[3] = {sH(s, 0), sH(s, 1), sH(s, 2)};
        // smem index of grid cell (j, k) in the E / H regions
        auto ei = [&](int j, int k) { return (j - j0 + 1) * EW + (k - k0 + HP); };
        auto hi = [&](int j, int k) { return (j - j0 + 1) * HW + (k - k0 + HP); };
        auto ni = [&](int j, int k) { return (j - j0 + 1) * NW + (k - k0 + 1); };

        // H^{n+1/2}(p) at (j, k); returns the three components
        auto h_at = [&](int j, int k, bool own, T &hx, T &hy, T &hz) {
            const bool interior = is_interior(p, j, k, nx, ny, nz, npml);
            const int e = ei(j, k);
            const T ex0 = E0[0][e], ey0 = E0[1][e], ez0 = E0[2][e];
            DE<T> d;
            if (interior) {
                d.zy = E0[2][e + EW] - ez0;
                d.yz = E0[1][e + 1] - ey0;
                d.xz = E0[0][e + 1] - ex0;
                d.zx = E1[2][e] - ez0;
                d.yx = E1[1][e] - ey0;
                d.xy = E0[0][e + EW] - ex0;
            } else {
                d.zy = (j < ny - 1) ? (E0[2][e + EW] - ez0) : T(0);
                d.yz = (k < nz - 1) ? (E0[1][e + 1] - ey0) : T(0);
                d.xz = (k < nz - 1) ? (E0[0][e + 1] - ex0) : T(0);
                d.zx = (p < nx - 1) ? (E1[2][e] - ez0) : T(0);
                d.yx = (p < nx - 1) ? (E1[1][e] - ey0) : T(0);
                d.xy = (j < ny - 1) ? (E0[0][e + EW] - ex0) : T(0);
            }
            const int h = hi(j, k);
            hx = H0[0][h];
            hy = H0[1][h];
            hz = H0[2][h];
            if (own && real_plane)
                h_cell<T, true>(interior, p, j, k, nx, ny, nz, npml, dtm, dtm_dl, d, a.cph,
                                a.psi_h, a.psi_h_next, hx, hy, hz);
            else
                h_cell<T, false>(interior, p, j, k, nx, ny, nz, npml, dtm, dtm_dl, d, a.cph,
                                 a.psi_h, a.psi_h_next, hx, hy, hz);
        };

        T own_h[RPT][3];
        const int k = k0 + tx;
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int j = j0 + ty * RPT + r;
            if (k < nz && j < ny) {
                h_at(j, k, true, own_h[r][0], own_h[r][1], own_h[r][2]);
                const int n = ni(j, k);
                sNew[0 * L::NW * L::NH + n] = own_h[r][0];
                sNew[1 * L::NW * L::NH + n] = own_h[r][1];
                sNew[2 * L::NW * L::NH + n] = own_h[r][2];
            }
        }
        if (real_plane) {
            // halo row j0-1 (k in tile) and halo column k0-1 (j in tile)
            if (tid < TK) {
                const int kh = k0 + tid, jh = j0 - 1;
                if (jh >= 0 && kh < nz) {
                    T hx, hy, hz;
                    h_at(jh, kh, false, hx, hy, hz);
                    const int n = ni(jh, kh);
                    sNew[0 * L::NW * L::NH + n] = hx;
                    sNew[1 * L::NW * L::NH + n] = hy;
                    sNew[2 * L::NW * L::NH + n] = hz;
                }
            } else if (tid < TK + TJ) {
                const int jh = j0 + (tid - TK), kh = k0 - 1;
                if (kh >= 0 && jh < ny) {
                    T hx, hy, hz;
                    h_at(jh, kh, false, hx, hy, hz);
                    const int n = ni(jh, kh);
                    sNew[0 * L::NW * L::NH + n] = hx;
                    sNew[1 * L::NW * L::NH + n] = hy;
                    sNew[2 * L::NW * L::NH + n] = hz;
                }
            }
        }
        __syncthreads();

        if (real_plane) {
            const T *NXp = sNew, *NYp = sNew + L::NW * L::NH, *NZp = sNew + 2 * L::NW * L::NH;
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int j = j0 + ty * RPT + r;
                if (k >= nz || j >= ny) continue;
                const bool interior = is_interior(p, j, k, nx, ny, nz, npml);
                const int n = ni(j, k);
                const T hx0 = own_h[r][0], hy0 = own_h[r][1], hz0 = own_h[r][2];
                DH<T> d;
                if (interior) {
                    d.zy = hz0 - NZp[n - NW];
                    d.yz = hy0 - NYp[n - 1];
                    d.xz = hx0 - NXp[n - 1];
                    d.zx = hz0 - carry_hz[r];
                    d.yx = hy0 - carry_hy[r];
                    d.xy = hx0 - NXp[n - NW];
                } else {
                    d.zy = (j > 0) ? (hz0 - NZp[n - NW]) : T(0);
                    d.yz = (k > 0) ? (hy0 - NYp[n - 1]) : T(0);
                    d.xz = (k > 0) ? (hx0 - NXp[n - 1]) : T(0);
                    d.zx = (p > 0) ? (hz0 - carry_hz[r]) : T(0);
                    d.yx = (p > 0) ? (hy0 - carry_hy[r]) : T(0);
                    d.xy = (j > 0) ? (hx0 - NXp[n - NW]) : T(0);
                }
                const int c = (j - j0) * TK + (k - k0);
                const int e = ei(j, k);
                const T cex = sC(s, 0)[c], cey = sC(s, 1)[c], cez = sC(s, 2)[c];
                T cax = T(1), cay = T(1), caz = T(1);
                if (LOSSY) {
                    cax = sA(s, 0)[c];
                    cay = sA(s, 1)[c];
                    caz = sA(s, 2)[c];
                }
                T ex = E0[0][e], ey = E0[1][e], ez = E0[2][e];
                if (src.n) ex = apply_sources<T>(src, p, j, k, ex, cex);
                e_cell<T, LOSSY>(interior, p, j, k, nx, ny, nz, npml, inv_dl, d, a.cpe, a.psi_e,
                                 cax, cay, caz, cex, cey, cez, ex, ey, ez);
                const int64_t idx = (int64_t)p * sx + (int64_t)j * sy + k;
                a.H_next[0][idx] = hx0;
                a.H_next[1][idx] = hy0;
                a.H_next[2][idx] = hz0;
                a.E_next[0][idx] = ex;
                a.E_next[1][idx] = ey;
                a.E_next[2][idx] = ez;
                if (planes.n) {
                    const double v[6] = {(double)ex, (double)ey, (double)ez,
                                         (double)hx0, (double)hy0, (double)hz0};
                    plane_dft_cell(planes, p, j, k, nx, ny, nz, v);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            carry_hy[r] = own_h[r][1];
            carry_hz[r] = own_h[r][2];
        }
        __syncthreads();  // stage s and sNew are free
        if (tid == 0 && p + NSTAGE <= plast) issue(p + NSTAGE);
    }
    if (!ok) {
        // drain: wait (bounded) for every stage that may still have copies in flight
        __syncthreads();
        if (tid == 0) {
            for (int p = pfirst; p <= plast; ++p) {
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
    int nx, ny, nz, elem, b0, b1;
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

bool make_map(CUtensorMap *out, const void *base, int nx, int ny, int nz, int elem, int b0,
              int b1) {
    MapKey key;
    memset(&key, 0, sizeof(key));
    key.base = base;
    key.nx = nx;
    key.ny = ny;
    key.nz = nz;
    key.elem = elem;
    key.b0 = b0;
    key.b1 = b1;
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
    CUresult r = fn(out, elem == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                    3, const_cast<void *>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    if (g_maps.size() > 4096) g_maps.clear();
    g_maps.emplace(key, *out);
    return true;
}

// Chunks along i: enough CTAs to fill ~2 per SM over whole waves, chunk >= 16 planes.
int choose_chunks(int tiles, int nx, int sms) {
    const int slots = 2 * sms;
    int best = 1;
    double best_score = -1.0;
    for (int c = 1; c <= 32; ++c) {
        const int len = (nx + c - 1) / c;
        if (len < 16 && c > 1) break;
        const double waves = (double)tiles * c / slots;
        const double fill = waves / ceil(waves);
        const double score = fill * (1.0 - 1.5 / (len + 1.5));
        if (score > best_score + 1e-9) {
            best_score = score;
            best = c;
        }
    }
    return best;
}

}  // namespace

template <typename T>
cudaError_t launch_step_fused(const YeeArgs<T> &a, const SourceList &src, const PlaneList &pl,
                              cudaStream_t st) {
    using L = FusedTile<T>;
    const int elem = (int)sizeof(T);
    // TMA needs 16-byte aligned row strides and base addresses.
    if (((int64_t)a.nz * elem) % 16 != 0) return cudaErrorNotSupported;
    for (int c = 0; c < 3; ++c) {
        const void *ptrs[5] = {a.E[c], a.H[c], a.ce[c], a.E_next[c], a.H_next[c]};
        for (const void *q : ptrs)
            if (reinterpret_cast<uintptr_t>(q) % 16 != 0) return cudaErrorNotSupported;
        if (a.lossy && reinterpret_cast<uintptr_t>(a.ca[c]) % 16 != 0) return cudaErrorNotSupported;
    }
    FusedMaps maps;
    memset(&maps, 0, sizeof(maps));
    for (int c = 0; c < 3; ++c) {
        if (!make_map(&maps.E[c], a.E[c], a.nx, a.ny, a.nz, elem, L::EW, L::EH) ||
            !make_map(&maps.H[c], a.H[c], a.nx, a.ny, a.nz, elem, L::HW, L::HH) ||
            !make_map(&maps.C[c], a.ce[c], a.nx, a.ny, a.nz, elem, L::TK, L::TJ))
            return cudaErrorNotSupported;
        if (a.lossy && !make_map(&maps.A[c], a.ca[c], a.nx, a.ny, a.nz, elem, L::TK, L::TJ))
            return cudaErrorNotSupported;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ntk = (a.nz + L::TK - 1) / L::TK;
    const int ntj = (a.ny + L::TJ - 1) / L::TJ;
    const int tiles = ntk * ntj;
    const int nchunk = choose_chunks(tiles, a.nx, sms);
    const int chunk = (a.nx + nchunk - 1) / nchunk;
    dim3 grid(tiles, (a.nx + chunk - 1) / chunk, 1);
    dim3 block(L::TK, L::NTY, 1);
    const size_t smem = L::smem_bytes(a.lossy != 0);
    cudaError_t e;
    if (a.lossy) {
        e = cudaFuncSetAttribute(k_step_fused<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e != cudaSuccess) return e;
        k_step_fused<T, true><<<grid, block, smem, st>>>(maps, a, src, pl, ntk, chunk);
    } else {
        e = cudaFuncSetAttribute(k_step_fused<T, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_step_fused<T, false><<<grid, block, smem, st>>>(maps, a, src, pl, ntk, chunk);
    }
    return cudaGetLastError();
}

template cudaError_t launch_step_fused<float>(const YeeArgs<float> &, const SourceList &,
                                              const PlaneList &, cudaStream_t);
template cudaError_t launch_step_fused<double>(const YeeArgs<double> &, const SourceList &,
                                               const PlaneList &, cudaStream_t);

int read_fused_error(int reset) {
    int v = 0;
    cudaMemcpyFromSymbol(&v, g_fused_error, sizeof(int));
    if (reset) {
        int z = 0;
        cudaMemcpyToSymbol(g_fused_error, &z, sizeof(int));
    }
    return v;
}

}  // namespace fdtd
