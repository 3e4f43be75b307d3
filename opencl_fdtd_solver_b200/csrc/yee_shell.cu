// CPML shell half-steps of the fused schedule.
//
// The fused step splits the grid into the interior box handled by the
// single-pass kernel (yee_fused.cu) and a shell around it handled here, one
// thread per cell:
//   k_shell_H : H^{n+1/2} of every cell outside the box [lo, hi)^3 (the CPML
//               slabs; the whole grid when there is no box), H read from H and
//               written to H_next, psi_H in place.  Runs first.
//   k_shell_E : E^{n+1} of every cell outside [lo+1, hi)^3 (the slabs plus the
//               first interior layer, whose H neighbours straddle the slab
//               boundary), reading the final H^{n+1/2} from H_next, writing
//               E_next, psi_E in place, with the sheet injections and plane
//               DFTs of those cells.  Runs after the interior kernel.
// Per-cell arithmetic is yee_cell.cuh (reference yee_update.cl), so each cell
// rounds exactly as in the split kernels.
//
// Shell enumeration: a flat cell index over three disjoint groups,
//   A: i outside [lo_x, hi_x)                      all (j, k)
//   B: i inside,  j outside [lo_y, hi_y)           all k
//   C: i inside,  j inside,  k outside [lo_z, hi_z)
// decoded with multiply-high divisions (consecutive threads take consecutive k).
#include <cuda_runtime.h>

#include "launch_count.cuh"
#include "yee_launch.cuh"

namespace fdtd {

// Unsigned 32-bit division by a divisor fixed at launch: a multiply-high and a
// shift in place of the runtime division sequence (Granlund & Montgomery,
// "Division by invariant integers using multiplication", PLDI 1994, round-up
// variant): with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (umulhi(m, n) + n) >> l for every 32-bit n, the sum taken in 64 bits.
struct FastDiv {
    unsigned d, m, l;
};

inline FastDiv make_fastdiv(unsigned d) {
    FastDiv f;
    f.d = d ? d : 1u;  // empty groups never divide
    f.l = 0;
    while ((1ull << f.l) < f.d) ++f.l;
    f.m = (unsigned)(((1ull << 32) * ((1ull << f.l) - f.d)) / f.d + 1ull);
    return f;
}

__device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv &f) {
    return (unsigned)(((unsigned long long)__umulhi(n, f.m) + n) >> f.l);
}

// Host-precomputed sizes of the three groups and their divisors.
struct ShellPlan {
    ShellBox b;
    int nax, nay, bx, by, cpr;  // slab planes in x, slab rows in y, box extents, C cells/row
    unsigned nA, nB, nC;        // cells per group
    FastDiv d_plane, d_nz, d_slab, d_cpr, d_by;  // ny*nz, nz, nay*nz, cpr, by
};

__device__ __forceinline__ bool shell_cell(unsigned t, int nx, int ny, int nz,
                                           const ShellPlan &s, int &i, int &j, int &k) {
    (void)nx;
    (void)ny;
    if (t < s.nA) {
        const unsigned q = fdiv(t, s.d_plane);
        const unsigned rem = t - q * s.d_plane.d;
        i = (int)q < s.b.lo[0] ? (int)q : s.b.hi[0] + ((int)q - s.b.lo[0]);
        const unsigned jj = fdiv(rem, s.d_nz);
        j = (int)jj;
        k = (int)(rem - jj * (unsigned)nz);
        return true;
    }
    t -= s.nA;
    if (t < s.nB) {
        const unsigned q = fdiv(t, s.d_slab);
        const unsigned rem = t - q * s.d_slab.d;
        i = s.b.lo[0] + (int)q;
        const unsigned r = fdiv(rem, s.d_nz);
        j = (int)r < s.b.lo[1] ? (int)r : s.b.hi[1] + ((int)r - s.b.lo[1]);
        k = (int)(rem - r * (unsigned)nz);
        return true;
    }
    t -= s.nB;
    if (t < s.nC) {
        const unsigned row = fdiv(t, s.d_cpr);
        const int c = (int)(t - row * (unsigned)s.cpr);
        const unsigned bi = fdiv(row, s.d_by);
        i = s.b.lo[0] + (int)bi;
        j = s.b.lo[1] + (int)(row - bi * (unsigned)s.by);
        k = c < s.b.lo[2] ? c : s.b.hi[2] + (c - s.b.lo[2]);
        return true;
    }
    return false;
}

ShellPlan make_plan(int nx, int ny, int nz, const ShellBox &b) {
    ShellPlan s;
    s.b = b;
    s.nax = b.lo[0] + (nx - b.hi[0]);
    s.nay = b.lo[1] + (ny - b.hi[1]);
    s.bx = b.hi[0] - b.lo[0];
    s.by = b.hi[1] - b.lo[1];
    s.cpr = b.lo[2] + (nz - b.hi[2]);
    s.nA = (unsigned)((int64_t)s.nax * ny * nz);
    s.nB = (unsigned)((int64_t)s.bx * s.nay * nz);
    s.nC = (unsigned)((int64_t)s.bx * s.by * s.cpr);
    s.d_plane = make_fastdiv((unsigned)ny * (unsigned)nz);
    s.d_nz = make_fastdiv((unsigned)nz);
    s.d_slab = make_fastdiv((unsigned)s.nay * (unsigned)nz);
    s.d_cpr = make_fastdiv((unsigned)(s.cpr > 0 ? s.cpr : 0));
    s.d_by = make_fastdiv((unsigned)(s.by > 0 ? s.by : 0));
    return s;
}

constexpr int SHELL_THREADS = 256;

template <typename T>
__global__ void __launch_bounds__(SHELL_THREADS)
    k_shell_H(YeeArgs<T> a, ShellPlan sp) {
    const int nx = a.nx, ny = a.ny, nz = a.nz, npml = a.npml;
    int i, j, k;
    if (!shell_cell(blockIdx.x * SHELL_THREADS + threadIdx.x, nx, ny, nz, sp, i, j, k)) return;
    const int64_t sx = (int64_t)ny * nz, sy = nz;
    const int64_t idx = (int64_t)i * sx + (int64_t)j * sy + k;
    const T *Ex = a.E[0], *Ey = a.E[1], *Ez = a.E[2];
    const bool interior = is_interior(i, j, k, nx, ny, nz, npml);
    const T ex0 = Ex[idx], ey0 = Ey[idx], ez0 = Ez[idx];
    DE<T> d;
    d.zy = (j < ny - 1) ? (Ez[idx + sy] - ez0) : T(0);
    d.yz = (k < nz - 1) ? (Ey[idx + 1] - ey0) : T(0);
    d.xz = (k < nz - 1) ? (Ex[idx + 1] - ex0) : T(0);
    d.zx = (i < nx - 1) ? (Ez[idx + sx] - ez0) : T(0);
    d.yx = (i < nx - 1) ? (Ey[idx + sx] - ey0) : T(0);
    d.xy = (j < ny - 1) ? (Ex[idx + sy] - ex0) : T(0);
    T hx = a.H[0][idx], hy = a.H[1][idx], hz = a.H[2][idx];
    h_cell<T, true>(interior, i, j, k, nx, ny, nz, npml, a.dtm, a.dtm_dl, d, a.cph, a.psi_h,
                    a.psi_h, hx, hy, hz);
    a.H_next[0][idx] = hx;
    a.H_next[1][idx] = hy;
    a.H_next[2][idx] = hz;
}

// planes points at the kernel's __grid_constant__ parameter, so the call takes
// no local copy of the descriptor list.
__device__ __noinline__ void shell_dft(const PlaneList *planes, int i, int j, int k, int nx,
                                       int ny, int nz, double ex, double ey, double ez,
                                       double hx, double hy, double hz) {
    const double v[6] = {ex, ey, ez, hx, hy, hz};
    plane_dft_cell(*planes, i, j, k, nx, ny, nz, v);
}

template <typename T, bool LOSSY>
__global__ void __launch_bounds__(SHELL_THREADS)
    k_shell_E(YeeArgs<T> a, ShellPlan sp, SourceList src, const __grid_constant__ PlaneList planes) {
    const int nx = a.nx, ny = a.ny, nz = a.nz, npml = a.npml;
    int i, j, k;
    if (!shell_cell(blockIdx.x * SHELL_THREADS + threadIdx.x, nx, ny, nz, sp, i, j, k)) return;
    const int64_t sx = (int64_t)ny * nz, sy = nz;
    const int64_t idx = (int64_t)i * sx + (int64_t)j * sy + k;
    const T *Hx = a.H_next[0], *Hy = a.H_next[1], *Hz = a.H_next[2];
    const bool interior = is_interior(i, j, k, nx, ny, nz, npml);
    const T hx0 = Hx[idx], hy0 = Hy[idx], hz0 = Hz[idx];
    DH<T> d;
    d.zy = (j > 0) ? (hz0 - Hz[idx - sy]) : T(0);
    d.yz = (k > 0) ? (hy0 - Hy[idx - 1]) : T(0);
    d.xz = (k > 0) ? (hx0 - Hx[idx - 1]) : T(0);
    d.zx = (i > 0) ? (hz0 - Hz[idx - sx]) : T(0);
    d.yx = (i > 0) ? (hy0 - Hy[idx - sx]) : T(0);
    d.xy = (j > 0) ? (hx0 - Hx[idx - sy]) : T(0);
    const T cex = a.ce[0][idx], cey = a.ce[1][idx], cez = a.ce[2][idx];
    T cax = T(1), cay = T(1), caz = T(1);
    if (LOSSY) {
        cax = a.ca[0][idx];
        cay = a.ca[1][idx];
        caz = a.ca[2][idx];
    }
    T ex = a.E[0][idx], ey = a.E[1][idx], ez = a.E[2][idx];
    if (src.n) ex = apply_sources<T>(src, i, j, k, ex, cex);
    e_cell<T, LOSSY>(interior, i, j, k, nx, ny, nz, npml, a.inv_dl, d, a.cpe, a.psi_e, cax, cay,
                     caz, cex, cey, cez, ex, ey, ez);
    a.E_next[0][idx] = ex;
    a.E_next[1][idx] = ey;
    a.E_next[2][idx] = ez;
    if (planes.n && plane_any_hit(planes, i, j, k))
        shell_dft(&planes, i, j, k, nx, ny, nz, (double)ex, (double)ey, (double)ez, (double)hx0,
                  (double)hy0, (double)hz0);
}

// One thread per cell of plane q inside box b: reads E^{n+1}, H^{n+1/2} of the
// cell from E_next / H_next and accumulates the plane's DFT (same arithmetic
// as the E epilogue, so the sums are identical).
template <typename T>
__global__ void __launch_bounds__(SHELL_THREADS)
    k_plane_dft_box(YeeArgs<T> a, ShellBox b, PlaneList planes, int q) {
    const fdtd_plane_dft &p = planes.p[q];
    const int ax = p.axis, u = (ax == 0) ? 1 : 0, w = (ax == 2) ? 1 : 2;
    const int nu = b.hi[u] - b.lo[u], nw = b.hi[w] - b.lo[w];
    const unsigned t = blockIdx.x * SHELL_THREADS + threadIdx.x;
    if (t >= (unsigned)nu * (unsigned)nw) return;
    int c[3];
    c[ax] = p.index;
    c[u] = b.lo[u] + (int)(t / (unsigned)nw);
    c[w] = b.lo[w] + (int)(t % (unsigned)nw);
    const int64_t idx = ((int64_t)c[0] * a.ny + c[1]) * a.nz + c[2];
    double v[6];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        v[m] = (p.comp_mask & (1 << m)) ? (double)a.E_next[m][idx] : 0.0;
        v[m + 3] = (p.comp_mask & (8 << m)) ? (double)a.H_next[m][idx] : 0.0;
    }
    PlaneList one;
    one.p[0] = p;
    one.n = 1;
    plane_dft_cell(one, c[0], c[1], c[2], a.nx, a.ny, a.nz, v);
}

template <typename T>
cudaError_t launch_plane_dft_box(const YeeArgs<T> &a, const ShellBox &b, const PlaneList &pl,
                                 cudaStream_t st) {
    for (int q = 0; q < pl.n; ++q) {
        const int ax = pl.p[q].axis, u = (ax == 0) ? 1 : 0, w = (ax == 2) ? 1 : 2;
        if (pl.p[q].index < b.lo[ax] || pl.p[q].index >= b.hi[ax]) continue;
        const int64_t n = (int64_t)(b.hi[u] - b.lo[u]) * (b.hi[w] - b.lo[w]);
        if (n <= 0) continue;
        k_plane_dft_box<T><<<(unsigned)((n + SHELL_THREADS - 1) / SHELL_THREADS), SHELL_THREADS, 0,
                             st>>>(a, b, pl, q);
        count_launches(1);
    }
    return cudaGetLastError();
}

template cudaError_t launch_plane_dft_box<float>(const YeeArgs<float> &, const ShellBox &,
                                                 const PlaneList &, cudaStream_t);
template cudaError_t launch_plane_dft_box<double>(const YeeArgs<double> &, const ShellBox &,
                                                  const PlaneList &, cudaStream_t);

static unsigned shell_blocks(const ShellPlan &s) {
    const uint64_t n = (uint64_t)s.nA + s.nB + s.nC;
    return (unsigned)((n + SHELL_THREADS - 1) / SHELL_THREADS);
}

static bool plan_fits(int nx, int ny, int nz, const ShellBox &b) {
    // every group count and the flat index must fit in 32 bits
    const int64_t nax = b.lo[0] + (nx - b.hi[0]), nay = b.lo[1] + (ny - b.hi[1]);
    const int64_t tot = nax * ny * nz + (int64_t)(b.hi[0] - b.lo[0]) * nay * nz +
                        (int64_t)(b.hi[0] - b.lo[0]) * (b.hi[1] - b.lo[1]) *
                            (b.lo[2] + (nz - b.hi[2]));
    return tot + SHELL_THREADS < 0xffffffffLL && (int64_t)ny * nz < 0xffffffffLL;
}

template <typename T>
cudaError_t launch_shell_H(const YeeArgs<T> &a, const ShellBox &b, cudaStream_t st) {
    if (!plan_fits(a.nx, a.ny, a.nz, b)) return cudaErrorInvalidConfiguration;
    const ShellPlan sp = make_plan(a.nx, a.ny, a.nz, b);
    const unsigned nb = shell_blocks(sp);
    if (nb == 0) return cudaSuccess;
    k_shell_H<T><<<nb, SHELL_THREADS, 0, st>>>(a, sp);
    count_launches(1);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_shell_E(const YeeArgs<T> &a, const ShellBox &b, const SourceList &src,
                           const PlaneList &pl, cudaStream_t st) {
    if (!plan_fits(a.nx, a.ny, a.nz, b)) return cudaErrorInvalidConfiguration;
    const ShellPlan sp = make_plan(a.nx, a.ny, a.nz, b);
    const unsigned nb = shell_blocks(sp);
    if (nb == 0) return cudaSuccess;
    if (a.lossy)
        k_shell_E<T, true><<<nb, SHELL_THREADS, 0, st>>>(a, sp, src, pl);
    else
        k_shell_E<T, false><<<nb, SHELL_THREADS, 0, st>>>(a, sp, src, pl);
    count_launches(1);
    return cudaGetLastError();
}

template cudaError_t launch_shell_H<float>(const YeeArgs<float> &, const ShellBox &, cudaStream_t);
template cudaError_t launch_shell_H<double>(const YeeArgs<double> &, const ShellBox &,
                                            cudaStream_t);
template cudaError_t launch_shell_E<float>(const YeeArgs<float> &, const ShellBox &,
                                           const SourceList &, const PlaneList &, cudaStream_t);
template cudaError_t launch_shell_E<double>(const YeeArgs<double> &, const ShellBox &,
                                            const SourceList &, const PlaneList &, cudaStream_t);

}  // namespace fdtd
