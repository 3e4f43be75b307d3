// Enumeration of the cells of an outer box that lie outside an inner box (the
// CPML shell around an interior box), one flat index per cell, shared by the
// forward shell kernels (yee_shell.cu) and the adjoint shell kernels
// (adjoint.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "yee_launch.cuh"

namespace fdtd {

constexpr int SHELL_THREADS = 256;

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

// Host-precomputed sizes of the three groups and their divisors.  The cells
// enumerated are those of the outer box o = [o.lo, o.hi) that lie outside the
// inner box b = [b.lo, b.hi) (b inside o; lo == hi on every axis means an empty
// inner box, so the whole outer box is enumerated).
struct ShellPlan {
    ShellBox b, o;
    int nax, nay, bx, by, cpr, oy, oz;  // slab planes in x, slab rows in y, inner extents,
                                        // C cells per row, outer extents in y and z
    unsigned nA, nB, nC;                // cells per group
    FastDiv d_plane, d_nz, d_slab, d_cpr, d_by;  // oy*oz, oz, nay*oz, cpr, by
};

__device__ __forceinline__ bool shell_cell(unsigned t, const ShellPlan &s, int &i, int &j,
                                           int &k) {
    const unsigned oz = (unsigned)s.oz;
    if (t < s.nA) {
        const unsigned q = fdiv(t, s.d_plane);
        const unsigned rem = t - q * s.d_plane.d;
        const int nlo = s.b.lo[0] - s.o.lo[0];
        i = (int)q < nlo ? s.o.lo[0] + (int)q : s.b.hi[0] + ((int)q - nlo);
        const unsigned jj = fdiv(rem, s.d_nz);
        j = s.o.lo[1] + (int)jj;
        k = s.o.lo[2] + (int)(rem - jj * oz);
        return true;
    }
    t -= s.nA;
    if (t < s.nB) {
        const unsigned q = fdiv(t, s.d_slab);
        const unsigned rem = t - q * s.d_slab.d;
        i = s.b.lo[0] + (int)q;
        const unsigned r = fdiv(rem, s.d_nz);
        const int nlo = s.b.lo[1] - s.o.lo[1];
        j = (int)r < nlo ? s.o.lo[1] + (int)r : s.b.hi[1] + ((int)r - nlo);
        k = s.o.lo[2] + (int)(rem - r * oz);
        return true;
    }
    t -= s.nB;
    if (t < s.nC) {
        const unsigned row = fdiv(t, s.d_cpr);
        const int c = (int)(t - row * (unsigned)s.cpr);
        const unsigned bi = fdiv(row, s.d_by);
        i = s.b.lo[0] + (int)bi;
        j = s.b.lo[1] + (int)(row - bi * (unsigned)s.by);
        const int nlo = s.b.lo[2] - s.o.lo[2];
        k = c < nlo ? s.o.lo[2] + c : s.b.hi[2] + (c - nlo);
        return true;
    }
    return false;
}

// An empty inner box (lo == hi == 0 on every axis) enumerates all of o.
inline ShellPlan make_plan(const ShellBox &o, const ShellBox &b) {
    ShellPlan s;
    s.o = o;
    s.b = b;
    if (b.lo[0] == b.hi[0] && b.lo[1] == b.hi[1] && b.lo[2] == b.hi[2])
        for (int d = 0; d < 3; ++d) s.b.lo[d] = s.b.hi[d] = o.lo[d];
    const ShellBox &B = s.b;
    s.oy = o.hi[1] - o.lo[1];
    s.oz = o.hi[2] - o.lo[2];
    s.nax = (B.lo[0] - o.lo[0]) + (o.hi[0] - B.hi[0]);
    s.nay = (B.lo[1] - o.lo[1]) + (o.hi[1] - B.hi[1]);
    s.bx = B.hi[0] - B.lo[0];
    s.by = B.hi[1] - B.lo[1];
    s.cpr = (B.lo[2] - o.lo[2]) + (o.hi[2] - B.hi[2]);
    s.nA = (unsigned)((int64_t)s.nax * s.oy * s.oz);
    s.nB = (unsigned)((int64_t)s.bx * s.nay * s.oz);
    s.nC = (unsigned)((int64_t)s.bx * s.by * s.cpr);
    s.d_plane = make_fastdiv((unsigned)s.oy * (unsigned)s.oz);
    s.d_nz = make_fastdiv((unsigned)s.oz);
    s.d_slab = make_fastdiv((unsigned)s.nay * (unsigned)s.oz);
    s.d_cpr = make_fastdiv((unsigned)(s.cpr > 0 ? s.cpr : 0));
    s.d_by = make_fastdiv((unsigned)(s.by > 0 ? s.by : 0));
    return s;
}

inline unsigned shell_blocks(const ShellPlan &s) {
    const uint64_t n = (uint64_t)s.nA + s.nB + s.nC;
    return (unsigned)((n + SHELL_THREADS - 1) / SHELL_THREADS);
}

// Enumeration of the cells of up to MAX_PLAN_BOXES disjoint boxes, one flat
// index per cell (box by box, k fastest), decoded with the same multiply-high
// divisions.
constexpr int MAX_PLAN_BOXES = 16;
struct BoxPlan {
    int n;
    ShellBox box[MAX_PLAN_BOXES];
    unsigned start[MAX_PLAN_BOXES + 1];                      // flat index of each box's first cell
    FastDiv d_plane[MAX_PLAN_BOXES], d_row[MAX_PLAN_BOXES];  // ey*ez, ez of each box
};

__device__ __forceinline__ bool box_cell(unsigned t, const BoxPlan &p, int &i, int &j, int &k) {
    if (t >= p.start[p.n]) return false;
    int b = 0;
    while (b + 1 < p.n && t >= p.start[b + 1]) ++b;
    t -= p.start[b];
    const unsigned q = fdiv(t, p.d_plane[b]);
    const unsigned rem = t - q * p.d_plane[b].d;
    const unsigned r = fdiv(rem, p.d_row[b]);
    i = p.box[b].lo[0] + (int)q;
    j = p.box[b].lo[1] + (int)r;
    k = p.box[b].lo[2] + (int)(rem - r * p.d_row[b].d);
    return true;
}

// Appends box [lo, hi) to the plan (empty boxes are skipped); false when the
// plan is full or the cell count would leave 32 bits.
inline bool plan_add(BoxPlan &p, int lo0, int hi0, int lo1, int hi1, int lo2, int hi2) {
    if (hi0 <= lo0 || hi1 <= lo1 || hi2 <= lo2) return true;
    if (p.n >= MAX_PLAN_BOXES) return false;
    const uint64_t cells = (uint64_t)(hi0 - lo0) * (hi1 - lo1) * (hi2 - lo2);
    if ((uint64_t)p.start[p.n] + cells + SHELL_THREADS >= 0xffffffffull) return false;
    ShellBox &b = p.box[p.n];
    b.lo[0] = lo0;
    b.hi[0] = hi0;
    b.lo[1] = lo1;
    b.hi[1] = hi1;
    b.lo[2] = lo2;
    b.hi[2] = hi2;
    p.d_plane[p.n] = make_fastdiv((unsigned)((hi1 - lo1) * (hi2 - lo2)));
    p.d_row[p.n] = make_fastdiv((unsigned)(hi2 - lo2));
    p.start[p.n + 1] = p.start[p.n] + (unsigned)cells;
    ++p.n;
    return true;
}

inline unsigned plan_blocks(const BoxPlan &p) {
    return (unsigned)(((uint64_t)p.start[p.n] + SHELL_THREADS - 1) / SHELL_THREADS);
}

// E^{n+1} of the cells of the plan's boxes (per-cell kernel, yee_shell.cu).
template <typename T>
cudaError_t launch_shell_E_boxes(const YeeArgs<T> &a, const BoxPlan &bp, const SourceList &src,
                                 const PlaneList &pl, cudaStream_t st);

inline bool plan_fits(const ShellBox &o) {
    // every group count and the flat index must fit in 32 bits
    const int64_t ex[3] = {o.hi[0] - o.lo[0], o.hi[1] - o.lo[1], o.hi[2] - o.lo[2]};
    return ex[0] * ex[1] * ex[2] + SHELL_THREADS < 0xffffffffLL;
}

inline ShellBox whole_grid(int nx, int ny, int nz) {
    ShellBox o;
    o.lo[0] = o.lo[1] = o.lo[2] = 0;
    o.hi[0] = nx;
    o.hi[1] = ny;
    o.hi[2] = nz;
    return o;
}

}  // namespace fdtd
