// extern "C" entry points of libfdtd_b200.so (declared in include/fdtd_b200.h):
// argument validation, dtype dispatch, status codes and error messages.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/fdtd_b200.h"
#include "yee_launch.cuh"
#include "adjoint.cuh"
#include "n2f.cuh"
#include "hostio.cuh"

namespace fdtd {
template <typename T>
cudaError_t launch_dft_faces(int nx, int ny, int nz, const T *const E[3], const T *const H[3],
                             const fdtd_box &b, double *acc, const double *phase,
                             cudaStream_t st);
int rel_change_blocks(int n);
cudaError_t launch_rel_change(const double *cur, const double *prev, int n, int nfreq, int fi,
                              double *scratch, double *out2, cudaStream_t st);
cudaError_t launch_farfield(const fdtd_box &b, const double *acc, int fi, double dl,
                            double k_wave, double eta0, const double *obs, int n_obs,
                            double *nl, double *eh, cudaStream_t st);
int read_fused_error(int reset);
void set_interior_wait_polls(int64_t polls);
cudaError_t launch_farfield_eh(const void *nl, int nl_f64, const double *obs, int n_obs,
                               double k_wave, double eta0, double *eh, cudaStream_t st);
void profile_enable(bool on);
cudaError_t profile_read(double ms[5], int *steps);
struct MatScalars {
    double scale, dt, two_eps0, eps0;
};
template <typename T, typename S>
cudaError_t launch_edge_coeffs(int nx, int ny, int nz, const S *eps, const S *sigma,
                               const MatScalars &m, T *const ce[3], T *const ca[3],
                               cudaStream_t st);

std::atomic<long long> g_launches{0};
void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
int noalloc_rel_max_face();
cudaError_t launch_rel_change_noalloc(const double *cur, const double *prev, int n, int nfreq,
                                      int fi, double *out2, cudaStream_t st);
}  // namespace fdtd

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return FDTD_OK;
    if (e == cudaErrorNotSupported)
        return fail(FDTD_ERR_UNSUPPORTED, "%s: not supported for this shape/alignment", what);
    return fail(FDTD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int check_grid(const fdtd_grid *g) {
    if (!g) return fail(FDTD_ERR_INVALID, "grid is NULL");
    if (g->nx <= 0 || g->ny <= 0 || g->nz <= 0)
        return fail(FDTD_ERR_INVALID, "grid shape must be positive, got (%d, %d, %d)", g->nx,
                    g->ny, g->nz);
    if (g->ny > 65535 * 8 || g->nx > 65535)
        return fail(FDTD_ERR_INVALID, "grid too large for the launch geometry (%d, %d, %d)",
                    g->nx, g->ny, g->nz);
    if (g->npml < 0) return fail(FDTD_ERR_INVALID, "npml must be >= 0, got %d", g->npml);
    if (g->dtype != FDTD_F32 && g->dtype != FDTD_F64)
        return fail(FDTD_ERR_INVALID, "dtype must be FDTD_F32 or FDTD_F64, got %d", g->dtype);
    if (g->x_slab) {
        if ((g->pml_x_lo != 0 && g->pml_x_lo != g->npml) ||
            (g->pml_x_hi != 0 && g->pml_x_hi != g->npml))
            return fail(FDTD_ERR_INVALID, "slab x-CPML layers (%d, %d) must each be 0 or npml=%d",
                        g->pml_x_lo, g->pml_x_hi, g->npml);
        if ((g->ghost_lo != 0 && g->ghost_lo != 1) || (g->ghost_hi != 0 && g->ghost_hi != 1))
            return fail(FDTD_ERR_INVALID, "slab ghost flags (%d, %d) must be 0 or 1", g->ghost_lo,
                        g->ghost_hi);
        if ((g->ghost_lo && g->pml_x_lo) || (g->ghost_hi && g->pml_x_hi))
            return fail(FDTD_ERR_INVALID, "a slab face is either a ghost or an x-CPML face");
        if (g->npml < 1)
            return fail(FDTD_ERR_INVALID, "a slab needs npml >= 1");
        if (g->nx < g->pml_x_lo + g->pml_x_hi + g->ghost_lo + g->ghost_hi + 1)
            return fail(FDTD_ERR_INVALID, "slab of %d planes is thinner than its CPML and ghosts",
                        g->nx);
    }
    return FDTD_OK;
}

// x CPML layers and interior x bounds of a grid or slab.
fdtd::XBounds x_bounds(const fdtd_grid *g) {
    fdtd::XBounds xb;
    if (g->x_slab) {
        // H's interior form reads E at x+1 (not on the upper ghost), E's reads H
        // at x-1 (not on the lower ghost)
        xb.pml_lo = g->pml_x_lo;
        xb.pml_hi = g->pml_x_hi;
        xb.h_lo = g->pml_x_lo;
        xb.h_hi = g->pml_x_hi > g->ghost_hi ? g->pml_x_hi : g->ghost_hi;
        xb.e_lo = g->pml_x_lo > g->ghost_lo ? g->pml_x_lo : g->ghost_lo;
        xb.e_hi = g->pml_x_hi;
    } else {
        xb.pml_lo = xb.pml_hi = xb.h_lo = xb.h_hi = xb.e_lo = xb.e_hi = g->npml;
    }
    return xb;
}

int check_fields(const fdtd_grid *g, const fdtd_fields *f, bool need_next) {
    if (!f) return fail(FDTD_ERR_INVALID, "fields is NULL");
    for (int c = 0; c < 3; ++c) {
        if (!f->E[c] || !f->H[c] || !f->ce[c])
            return fail(FDTD_ERR_INVALID, "field/coefficient pointer %d is NULL", c);
        if (g->lossy && !f->ca[c]) return fail(FDTD_ERR_INVALID, "lossy grid without ca[%d]", c);
        if (need_next) {
            if (!f->E_next[c] || !f->H_next[c])
                return fail(FDTD_ERR_INVALID, "E_next/H_next[%d] is NULL", c);
            if (f->E_next[c] == f->E[c] || f->H_next[c] == f->H[c])
                return fail(FDTD_ERR_INVALID, "fused step outputs must not alias inputs");
        }
    }
    return FDTD_OK;
}

int check_cpml(const fdtd_grid *g, const fdtd_cpml *c) {
    if (!c) return fail(FDTD_ERR_INVALID, "cpml is NULL");
    for (int a = 0; a < 3; ++a)
        if (!c->b_h[a] || !c->c_h[a] || !c->ik_h[a] || !c->b_e[a] || !c->c_e[a] || !c->ik_e[a])
            return fail(FDTD_ERR_INVALID, "CPML profile pointer for axis %d is NULL", a);
    if (g->npml > 0)
        for (int q = 0; q < 6; ++q) {
            if (!c->psi_h[q] || !c->psi_e[q])
                return fail(FDTD_ERR_INVALID, "psi stripe %d is NULL", q);
        }
    return FDTD_OK;
}

int build_sources(const fdtd_grid *g, const fdtd_source *src, int nsrc, fdtd::SourceList &out) {
    if (nsrc < 0 || nsrc > FDTD_MAX_SOURCES)
        return fail(FDTD_ERR_INVALID, "nsrc must be in [0, %d], got %d", FDTD_MAX_SOURCES, nsrc);
    if (nsrc > 0 && !src) return fail(FDTD_ERR_INVALID, "sources is NULL");
    memset(&out, 0, sizeof(out));
    out.n = nsrc;
    for (int q = 0; q < nsrc; ++q) {
        const fdtd_source &s = src[q];
        if (s.kind != FDTD_SRC_JX && s.kind != FDTD_SRC_EX)
            return fail(FDTD_ERR_INVALID, "source %d: unknown kind %d", q, s.kind);
        if (s.z < 0 || s.z >= g->nz)
            return fail(FDTD_ERR_INVALID, "source %d: z=%d outside [0, %d)", q, s.z, g->nz);
        out.s[q] = s;
    }
    return FDTD_OK;
}

int build_planes(const fdtd_grid *g, const fdtd_plane_dft *pl, int np, fdtd::PlaneList &out) {
    if (np < 0 || np > FDTD_MAX_PLANES)
        return fail(FDTD_ERR_INVALID, "nplanes must be in [0, %d], got %d", FDTD_MAX_PLANES, np);
    if (np > 0 && !pl) return fail(FDTD_ERR_INVALID, "planes is NULL");
    memset(&out, 0, sizeof(out));
    out.n = np;
    const int dims[3] = {g->nx, g->ny, g->nz};
    for (int q = 0; q < np; ++q) {
        const fdtd_plane_dft &p = pl[q];
        if (p.axis < 0 || p.axis > 2) return fail(FDTD_ERR_INVALID, "plane %d: axis %d", q, p.axis);
        if (p.index < 0 || p.index >= dims[p.axis])
            return fail(FDTD_ERR_INVALID, "plane %d: index %d outside [0, %d)", q, p.index,
                        dims[p.axis]);
        if (p.nfreq <= 0 || p.nfreq > FDTD_MAX_FREQS)
            return fail(FDTD_ERR_INVALID, "plane %d: nfreq %d outside [1, %d]", q, p.nfreq,
                        FDTD_MAX_FREQS);
        if ((p.comp_mask & 0x3f) == 0 || (p.comp_mask & ~0x3f))
            return fail(FDTD_ERR_INVALID, "plane %d: comp_mask 0x%x", q, p.comp_mask);
        if (!p.acc || !p.phase) return fail(FDTD_ERR_INVALID, "plane %d: NULL buffer", q);
        out.p[q] = p;
    }
    return FDTD_OK;
}

template <typename T>
fdtd::YeeArgs<T> make_args(const fdtd_grid *g, const fdtd_fields *f, const fdtd_cpml *c) {
    fdtd::YeeArgs<T> a;
    memset(&a, 0, sizeof(a));
    a.nx = g->nx;
    a.ny = g->ny;
    a.nz = g->nz;
    a.npml = g->npml;
    a.lossy = g->lossy ? 1 : 0;
    a.xb = x_bounds(g);
    a.ghost_lo = g->x_slab ? g->ghost_lo : 0;
    a.ghost_hi = g->x_slab ? g->ghost_hi : 0;
    a.dtm = (T)g->dtm;
    a.dtm_dl = (T)g->dtm_dl;
    a.inv_dl = (T)g->inv_dl;
    for (int q = 0; q < 3; ++q) {
        a.E[q] = (T *)f->E[q];
        a.H[q] = (T *)f->H[q];
        a.E_next[q] = (T *)f->E_next[q];
        a.H_next[q] = (T *)f->H_next[q];
        a.ce[q] = (const T *)f->ce[q];
        a.ca[q] = (const T *)f->ca[q];
        a.cph.b[q] = (const T *)c->b_h[q];
        a.cph.c[q] = (const T *)c->c_h[q];
        a.cph.ik[q] = (const T *)c->ik_h[q];
        a.cpe.b[q] = (const T *)c->b_e[q];
        a.cpe.c[q] = (const T *)c->c_e[q];
        a.cpe.ik[q] = (const T *)c->ik_e[q];
    }
    for (int q = 0; q < 6; ++q) {
        a.psi_h[q] = (T *)c->psi_h[q];
        a.psi_h_next[q] = (T *)c->psi_h_next[q];
        a.psi_e[q] = (T *)c->psi_e[q];
    }
    return a;
}

int check_box(const fdtd_grid *g, const fdtd_box *b) {
    if (!b) return fail(FDTD_ERR_INVALID, "box is NULL");
    if (g && (b->ix0 < 0 || b->ix1 >= g->nx || b->ix0 > b->ix1 || b->iy0 < 0 || b->iy1 >= g->ny ||
        b->iy0 > b->iy1 || b->iz0 < 0 || b->iz1 >= g->nz || b->iz0 > b->iz1))
        return fail(FDTD_ERR_INVALID, "box (%d..%d, %d..%d, %d..%d) outside the grid", b->ix0,
                    b->ix1, b->iy0, b->iy1, b->iz0, b->iz1);
    if (b->ix0 > b->ix1 || b->iy0 > b->iy1 || b->iz0 > b->iz1)
        return fail(FDTD_ERR_INVALID, "box is empty");
    const int64_t nxf = b->ix1 - b->ix0 + 1, nyf = b->iy1 - b->iy0 + 1, nzf = b->iz1 - b->iz0 + 1;
    const int64_t cnt[6] = {nyf * nzf, nyf * nzf, nxf * nzf, nxf * nzf, nxf * nyf, nxf * nyf};
    int64_t o = 0;
    for (int q = 0; q < 6; ++q) {
        if (b->off[q] != o) return fail(FDTD_ERR_INVALID, "box face offset %d is %d, expected %lld",
                                        q, b->off[q], (long long)o);
        o += cnt[q];
    }
    if (b->n_face != o) return fail(FDTD_ERR_INVALID, "box n_face %d, expected %lld", b->n_face,
                                    (long long)o);
    if (b->nfreq <= 0 || b->nfreq > FDTD_MAX_FREQS)
        return fail(FDTD_ERR_INVALID, "box nfreq %d outside [1, %d]", b->nfreq, FDTD_MAX_FREQS);
    return FDTD_OK;
}

// ---- adjoint --------------------------------------------------------------
int check_adjoint(const fdtd_grid *g, const fdtd_adjoint_fields *a) {
    if (!a) return fail(FDTD_ERR_INVALID, "adjoint fields is NULL");
    if (g->x_slab)
        return fail(FDTD_ERR_UNSUPPORTED, "the adjoint sweep runs on a whole grid, not a slab");
    if (g->lossy)
        return fail(FDTD_ERR_UNSUPPORTED, "the adjoint sweep needs a lossless grid (ca == 1)");
    for (int c = 0; c < 3; ++c)
        if (!a->E[c] || !a->H[c] || !a->ce[c])
            return fail(FDTD_ERR_INVALID, "adjoint field/coefficient pointer %d is NULL", c);
    if (g->npml > 0)
        for (int q = 0; q < 6; ++q) {
            if (!a->pe[q] || !a->pe_next[q] || !a->ph[q] || !a->ph_next[q])
                return fail(FDTD_ERR_INVALID, "adjoint P stripe %d is NULL", q);
            if (a->pe[q] == a->pe_next[q] || a->ph[q] == a->ph_next[q])
                return fail(FDTD_ERR_INVALID, "adjoint P stripe %d: next must not alias", q);
        }
    return FDTD_OK;
}

int build_seed(const fdtd_grid *g, const fdtd_adjoint_seed *s, fdtd::AdjSeed &out) {
    memset(&out, 0, sizeof(out));
    if (!s) return FDTD_OK;
    const int dims[3] = {g->nx, g->ny, g->nz};
    if (s->axis < 0 || s->axis > 2) return fail(FDTD_ERR_INVALID, "seed axis %d", s->axis);
    if (s->index < 0 || s->index >= dims[s->axis])
        return fail(FDTD_ERR_INVALID, "seed plane index %d outside [0, %d)", s->index,
                    dims[s->axis]);
    const int da = s->axis == 0 ? dims[1] : dims[0];
    const int db = s->axis == 2 ? dims[1] : dims[2];
    if (s->a0 < 0 || s->a1 > da || s->a0 >= s->a1 || s->b0 < 0 || s->b1 > db || s->b0 >= s->b1)
        return fail(FDTD_ERR_INVALID, "seed patch [%d,%d)x[%d,%d) is empty or outside the %dx%d plane",
                    s->a0, s->a1, s->b0, s->b1, da, db);
    if (s->comp_mask <= 0 || s->comp_mask > 7)
        return fail(FDTD_ERR_INVALID, "seed comp_mask 0x%x (E components only)", s->comp_mask);
    if (s->nfreq < 1 || s->nfreq > FDTD_MAX_FREQS)
        return fail(FDTD_ERR_INVALID, "seed nfreq %d outside [1, %d]", s->nfreq, FDTD_MAX_FREQS);
    if (!s->seed || !s->phase) return fail(FDTD_ERR_INVALID, "seed/phase is NULL");
    out.active = 1;
    out.axis = s->axis;
    out.index = s->index;
    out.a0 = s->a0;
    out.a1 = s->a1;
    out.b0 = s->b0;
    out.b1 = s->b1;
    out.comp_mask = s->comp_mask;
    out.nfreq = s->nfreq;
    out.seed = s->seed;
    out.phase = s->phase;
    return FDTD_OK;
}

int check_span(const fdtd_grid *g, const int32_t lo[3], const int32_t hi[3], const char *what) {
    const int dims[3] = {g->nx, g->ny, g->nz};
    for (int a = 0; a < 3; ++a)
        if (lo[a] < 0 || hi[a] > dims[a] || lo[a] >= hi[a])
            return fail(FDTD_ERR_INVALID, "%s axis %d: [%d, %d) is empty or outside [0, %d)", what,
                        a, lo[a], hi[a], dims[a]);
    return FDTD_OK;
}

template <typename T>
fdtd::AdjArgs<T> make_adj(const fdtd_grid *g, const fdtd_adjoint_fields *f, const fdtd_cpml *c) {
    fdtd::AdjArgs<T> a;
    memset(&a, 0, sizeof(a));
    a.nx = g->nx;
    a.ny = g->ny;
    a.nz = g->nz;
    a.npml = g->npml;
    a.dtm = (T)g->dtm;
    a.ik_int = (T)g->inv_dl;
    for (int q = 0; q < 3; ++q) {
        a.E[q] = (T *)f->E[q];
        a.H[q] = (T *)f->H[q];
        a.ce[q] = (const T *)f->ce[q];
        a.cph.b[q] = (const T *)c->b_h[q];
        a.cph.c[q] = (const T *)c->c_h[q];
        a.cph.ik[q] = (const T *)c->ik_h[q];
        a.cpe.b[q] = (const T *)c->b_e[q];
        a.cpe.c[q] = (const T *)c->c_e[q];
        a.cpe.ik[q] = (const T *)c->ik_e[q];
    }
    for (int q = 0; q < 6; ++q) {
        a.pe[q] = (const T *)f->pe[q];
        a.pe_next[q] = (T *)f->pe_next[q];
        a.ph[q] = (const T *)f->ph[q];
        a.ph_next[q] = (T *)f->ph_next[q];
    }
    return a;
}

template <typename T>
fdtd::AdjOut<T> adj_out(const fdtd_adjoint_fields *f) {
    fdtd::AdjOut<T> o;
    for (int q = 0; q < 3; ++q) {
        o.E[q] = (T *)f->E_next[q];
        o.H[q] = (T *)f->H_next[q];
    }
    return o;
}

template <typename T>
fdtd::AdjGrad<T> make_grad(const fdtd_grad_box *gb) {
    fdtd::AdjGrad<T> r;
    memset(&r, 0, sizeof(r));
    if (!gb) return r;
    r.active = 1;
    for (int q = 0; q < 3; ++q) {
        r.lo[q] = gb->lo[q];
        r.hi[q] = gb->hi[q];
    }
    r.e_next = (const T *)gb->e_next;
    r.e_prev = (const T *)gb->e_prev;
    r.g = gb->g;
    return r;
}

// ---- near-to-far contraction ------------------------------------------------
struct N2FPlan {
    fdtd::n2f::Params P;
    uint64_t btile_bytes, partial_off, total;
};

int plan_n2f(const fdtd_n2f_face *faces, int nfaces, int nfreq, int n_obs, int mode, N2FPlan &pl) {
    if (!faces) return fail(FDTD_ERR_INVALID, "faces is NULL");
    if (nfaces < 1 || nfaces > 6) return fail(FDTD_ERR_INVALID, "nfaces %d outside [1, 6]", nfaces);
    if (nfreq < 1 || nfreq > 65535) return fail(FDTD_ERR_INVALID, "nfreq %d outside [1, 65535]", nfreq);
    if (n_obs < 1) return fail(FDTD_ERR_INVALID, "n_obs must be positive, got %d", n_obs);
    if (mode != FDTD_N2F_BF16X3 && mode != FDTD_N2F_TF32 && mode != FDTD_N2F_FP64)
        return fail(FDTD_ERR_INVALID, "unknown near-to-far mode %d", mode);
    memset(&pl, 0, sizeof(pl));
    auto &P = pl.P;
    P.n_obs = n_obs;
    P.nfaces = nfaces;
    const bool tc = mode != FDTD_N2F_FP64;
    const int kr = tc ? fdtd::n2f::k_real_per_step(mode) : 16;
    const int64_t bcopy = tc ? fdtd::n2f::b_copy_bytes(mode) : 0;
    uint64_t off = 0;
    for (int f = 0; f < nfaces; ++f) {
        const fdtd_n2f_face &F = faces[f];
        if (F.normal < 0 || F.normal > 2)
            return fail(FDTD_ERR_INVALID, "face %d: normal axis %d", f, F.normal);
        if (F.np < 1 || F.nq < 1 || F.np > (1 << 20) || F.nq > (1 << 20))
            return fail(FDTD_ERR_INVALID, "face %d: sample counts %d x %d", f, F.np, F.nq);
        if (!F.cur) return fail(FDTD_ERR_INVALID, "face %d: cur is NULL", f);
        if (!(F.pitch > 0)) return fail(FDTD_ERR_INVALID, "face %d: pitch must be positive", f);
        auto &G = P.face[f];
        G.axis_n = F.normal;
        G.axis_p = F.normal == 0 ? 1 : 0;
        G.axis_q = F.normal == 2 ? 1 : 2;
        G.np = F.np;
        G.nq = F.nq;
        G.ks = (2 * F.np + kr - 1) / kr;
        G.nt = (F.nq + fdtd::n2f::QT - 1) / fdtd::n2f::QT;
        G.x_n = F.x_n;
        G.o_p = F.o_p;
        G.o_q = F.o_q;
        G.pitch = F.pitch;
        G.b_freq_stride = (int64_t)G.ks * G.nt * bcopy;
        G.b_off = (int64_t)off;
        off += (uint64_t)G.b_freq_stride * nfreq;
        P.cur[f] = F.cur;
        const int map[4] = {G.axis_p, G.axis_q, 3 + G.axis_p, 3 + G.axis_q};
        for (int c = 0; c < 4; ++c) P.comp_map[f * 4 + c] = map[c];
    }
    pl.btile_bytes = off;
    pl.partial_off = (off + 255) & ~(uint64_t)255;
    pl.total = tc ? pl.partial_off + (uint64_t)nfreq * nfaces * n_obs * 4 * 8 : 0;
    return FDTD_OK;
}

}  // namespace

extern "C" {

const char *fdtd_last_error(void) { return g_err.c_str(); }

const char *fdtd_version(void) { return "fdtd_b200 0.1 sm_100a"; }

int fdtd_device_status(int32_t *flags, int32_t reset) {
    if (!flags) return fail(FDTD_ERR_INVALID, "flags is NULL");
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_status(e, "device_status");
    *flags = fdtd::read_fused_error(reset) | (fdtd::n2f::read_error(reset) ? 2 : 0) |
             (fdtd::read_adjoint_error(reset) ? 4 : 0);
    return cuda_status(cudaGetLastError(), "device_status");
}

int fdtd_set_wait_budget(int32_t kernel, int64_t budget) {
    if (kernel == FDTD_WAIT_INTERIOR)
        fdtd::set_interior_wait_polls(budget);
    else if (kernel == FDTD_WAIT_N2F)
        fdtd::n2f::set_wait_ns(budget);
    else
        return fail(FDTD_ERR_INVALID, "unknown wait-budget kernel %d", kernel);
    return FDTD_OK;
}

int fdtd_update_H(const fdtd_grid *g, const fdtd_fields *f, const fdtd_cpml *c, void *stream) {
    int rc;
    if ((rc = check_grid(g)) || (rc = check_fields(g, f, false)) || (rc = check_cpml(g, c)))
        return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (g->dtype == FDTD_F32)
        return cuda_status(fdtd::launch_update_H<float>(make_args<float>(g, f, c), st), "update_H");
    return cuda_status(fdtd::launch_update_H<double>(make_args<double>(g, f, c), st), "update_H");
}

int fdtd_update_E(const fdtd_grid *g, const fdtd_fields *f, const fdtd_cpml *c,
                  const fdtd_source *src, int32_t nsrc, const fdtd_plane_dft *planes,
                  int32_t nplanes, void *stream) {
    int rc;
    if ((rc = check_grid(g)) || (rc = check_fields(g, f, false)) || (rc = check_cpml(g, c)))
        return rc;
    fdtd::SourceList sl;
    fdtd::PlaneList pl;
    if ((rc = build_sources(g, src, nsrc, sl)) || (rc = build_planes(g, planes, nplanes, pl)))
        return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (g->dtype == FDTD_F32)
        return cuda_status(fdtd::launch_update_E<float>(make_args<float>(g, f, c), sl, pl, st),
                           "update_E");
    return cuda_status(fdtd::launch_update_E<double>(make_args<double>(g, f, c), sl, pl, st),
                       "update_E");
}

int fdtd_step(const fdtd_grid *g, const fdtd_fields *f, const fdtd_cpml *c,
              const fdtd_source *src, int32_t nsrc, const fdtd_plane_dft *planes,
              int32_t nplanes, void *stream) {
    int rc;
    if ((rc = check_grid(g)) || (rc = check_fields(g, f, true)) || (rc = check_cpml(g, c)))
        return rc;
    fdtd::SourceList sl;
    fdtd::PlaneList pl;
    if ((rc = build_sources(g, src, nsrc, sl)) || (rc = build_planes(g, planes, nplanes, pl)))
        return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (g->dtype == FDTD_F32)
        return cuda_status(fdtd::launch_step_fused<float>(make_args<float>(g, f, c), sl, pl, st),
                           "step");
    return cuda_status(fdtd::launch_step_fused<double>(make_args<double>(g, f, c), sl, pl, st),
                       "step");
}

int fdtd_add_source(const fdtd_grid *g, void *Ex, const void *ce_x, const fdtd_source *src,
                    void *stream) {
    int rc;
    if ((rc = check_grid(g))) return rc;
    if (!Ex || !ce_x) return fail(FDTD_ERR_INVALID, "Ex/ce_x is NULL");
    fdtd::SourceList sl;
    if ((rc = build_sources(g, src, 1, sl))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (g->dtype == FDTD_F32)
        return cuda_status(fdtd::launch_add_source<float>(g->nx, g->ny, g->nz, *src, (float *)Ex,
                                                          (const float *)ce_x, st),
                           "add_source");
    return cuda_status(fdtd::launch_add_source<double>(g->nx, g->ny, g->nz, *src, (double *)Ex,
                                                       (const double *)ce_x, st),
                       "add_source");
}

int fdtd_dft_faces(const fdtd_grid *g, const void *const E[3], const void *const H[3],
                   const fdtd_box *box, double *acc, const double *phase, void *stream) {
    int rc;
    if ((rc = check_grid(g)) || (rc = check_box(g, box))) return rc;
    if (!E || !H || !acc || !phase) return fail(FDTD_ERR_INVALID, "NULL buffer");
    for (int q = 0; q < 3; ++q)
        if (!E[q] || !H[q]) return fail(FDTD_ERR_INVALID, "NULL field %d", q);
    cudaStream_t st = (cudaStream_t)stream;
    if (g->dtype == FDTD_F32) {
        const float *e[3] = {(const float *)E[0], (const float *)E[1], (const float *)E[2]};
        const float *h[3] = {(const float *)H[0], (const float *)H[1], (const float *)H[2]};
        return cuda_status(fdtd::launch_dft_faces<float>(g->nx, g->ny, g->nz, e, h, *box, acc,
                                                         phase, st),
                           "dft_faces");
    }
    const double *e[3] = {(const double *)E[0], (const double *)E[1], (const double *)E[2]};
    const double *h[3] = {(const double *)H[0], (const double *)H[1], (const double *)H[2]};
    return cuda_status(
        fdtd::launch_dft_faces<double>(g->nx, g->ny, g->nz, e, h, *box, acc, phase, st),
        "dft_faces");
}

int fdtd_rel_change_blocks(int32_t n_face) { return fdtd::rel_change_blocks(n_face); }

int fdtd_dft_rel_change(const double *cur, const double *prev, int32_t n_face, int32_t nfreq,
                        int32_t fi, double *scratch, double *out2, void *stream) {
    if (!cur || !prev || !scratch || !out2) return fail(FDTD_ERR_INVALID, "NULL buffer");
    if (n_face <= 0 || nfreq <= 0 || fi < 0 || fi >= nfreq)
        return fail(FDTD_ERR_INVALID, "n_face %d, nfreq %d, fi %d", n_face, nfreq, fi);
    return cuda_status(fdtd::launch_rel_change(cur, prev, n_face, nfreq, fi, scratch, out2,
                                               (cudaStream_t)stream),
                       "dft_rel_change");
}

int fdtd_dft_rel_change_noalloc(const double *cur, const double *prev, int32_t n_face,
                                int32_t nfreq, int32_t fi, double *out2, void *stream) {
    if (!cur || !prev || !out2) return fail(FDTD_ERR_INVALID, "NULL buffer");
    if (n_face <= 0 || nfreq <= 0 || fi < 0 || fi >= nfreq)
        return fail(FDTD_ERR_INVALID, "n_face %d, nfreq %d, fi %d", n_face, nfreq, fi);
    if (n_face > fdtd::noalloc_rel_max_face())
        return fail(FDTD_ERR_INVALID,
                    "n_face %d exceeds the %d face samples the built-in scratch array holds; "
                    "use fdtd_dft_rel_change with a caller buffer",
                    n_face, fdtd::noalloc_rel_max_face());
    return cuda_status(
        fdtd::launch_rel_change_noalloc(cur, prev, n_face, nfreq, fi, out2, (cudaStream_t)stream),
        "dft_rel_change_noalloc");
}

int fdtd_farfield(const fdtd_box *box, const double *acc, int32_t fi, double dl, double k_wave,
                  double eta0, const double *obs_xyz, int32_t n_obs, double *nl_scratch,
                  double *eh, void *stream) {
    if (!box || !acc || !obs_xyz || !nl_scratch || !eh)
        return fail(FDTD_ERR_INVALID, "NULL buffer");
    int rc;
    if ((rc = check_box(nullptr, box))) return rc;
    if (n_obs <= 0) return fail(FDTD_ERR_INVALID, "n_obs must be positive, got %d", n_obs);
    if (fi < 0 || fi >= box->nfreq)
        return fail(FDTD_ERR_INVALID, "frequency index %d outside [0, %d)", fi, box->nfreq);
    if (!(dl > 0) || !(k_wave >= 0) || !(eta0 > 0))
        return fail(FDTD_ERR_INVALID, "dl, k_wave, eta0 must be positive");
    return cuda_status(fdtd::launch_farfield(*box, acc, fi, dl, k_wave, eta0, obs_xyz, n_obs,
                                             nl_scratch, eh, (cudaStream_t)stream),
                       "farfield");
}

int fdtd_capture_box(const fdtd_grid *g, const void *const E[3], const int32_t lo[3],
                     const int32_t hi[3], void *out, void *stream) {
    int rc;
    if ((rc = check_grid(g))) return rc;
    if (!E || !E[0] || !E[1] || !E[2] || !out || !lo || !hi)
        return fail(FDTD_ERR_INVALID, "NULL buffer");
    if ((rc = check_span(g, lo, hi, "capture box"))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (g->dtype == FDTD_F32)
        return cuda_status(fdtd::launch_capture<float>(g->ny, g->nz, (const float *const *)E, lo,
                                                       hi, (float *)out, st),
                           "capture_box");
    return cuda_status(fdtd::launch_capture<double>(g->ny, g->nz, (const double *const *)E, lo,
                                                    hi, (double *)out, st),
                       "capture_box");
}

int fdtd_read_regions(const void *field, int32_t dtype, int32_t nx, int32_t ny, int32_t nz,
                      const fdtd_region *regions, int32_t nreg, void *staging, void *host,
                      void *stream) {
    if (dtype != FDTD_F32 && dtype != FDTD_F64) return fail(FDTD_ERR_INVALID, "dtype %d", dtype);
    if (nx <= 0 || ny <= 0 || nz <= 0)
        return fail(FDTD_ERR_INVALID, "shape (%d, %d, %d)", nx, ny, nz);
    if (nreg < 0 || nreg > FDTD_MAX_REGIONS)
        return fail(FDTD_ERR_INVALID, "%d regions (at most %d)", nreg, FDTD_MAX_REGIONS);
    if (nreg > 0 && !regions) return fail(FDTD_ERR_INVALID, "regions is NULL");
    const int dims[3] = {nx, ny, nz};
    fdtd::RegionList r;
    memset(&r, 0, sizeof(r));
    r.n = nreg;
    r.off[0] = 0;
    for (int q = 0; q < nreg; ++q) {
        int64_t cells = 1;
        for (int a = 0; a < 3; ++a) {
            const int32_t lo = regions[q].lo[a], hi = regions[q].hi[a];
            if (lo < 0 || hi > dims[a] || lo > hi)
                return fail(FDTD_ERR_INVALID, "region %d axis %d: [%d, %d) outside [0, %d)", q,
                            a, lo, hi, dims[a]);
            r.lo[q][a] = lo;
            r.ext[q][a] = hi - lo;
            cells *= hi - lo;
        }
        r.off[q + 1] = r.off[q] + cells;
    }
    if (r.off[nreg] == 0) return FDTD_OK;
    if (!field || !staging || !host) return fail(FDTD_ERR_INVALID, "NULL buffer");
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == FDTD_F32)
        return cuda_status(fdtd::launch_read_regions<float>((const float *)field, ny, nz, r,
                                                            (float *)staging, host, st),
                           "read_regions");
    return cuda_status(fdtd::launch_read_regions<double>((const double *)field, ny, nz, r,
                                                         (double *)staging, host, st),
                       "read_regions");
}

int fdtd_adjoint_seed_add(const fdtd_grid *g, void *const Ebar[3], const fdtd_adjoint_seed *seed,
                          void *stream) {
    int rc;
    if ((rc = check_grid(g))) return rc;
    if (!Ebar || !Ebar[0] || !Ebar[1] || !Ebar[2] || !seed)
        return fail(FDTD_ERR_INVALID, "NULL buffer");
    fdtd::AdjSeed sd;
    if ((rc = build_seed(g, seed, sd))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (g->dtype == FDTD_F32)
        return cuda_status(fdtd::launch_adjoint_seed<float>(g->nx, g->ny, g->nz,
                                                            (float *const *)Ebar, sd, st),
                           "adjoint_seed_add");
    return cuda_status(fdtd::launch_adjoint_seed<double>(g->nx, g->ny, g->nz,
                                                         (double *const *)Ebar, sd, st),
                       "adjoint_seed_add");
}

int fdtd_adjoint_step(const fdtd_grid *g, const fdtd_adjoint_fields *a, const fdtd_cpml *c,
                      const fdtd_grad_box *gb, const fdtd_adjoint_seed *next_seed,
                      void *stream) {
    int rc;
    if ((rc = check_grid(g)) || (rc = check_adjoint(g, a))) return rc;
    if (!c) return fail(FDTD_ERR_INVALID, "cpml is NULL");
    for (int q = 0; q < 3; ++q)
        if (!c->b_h[q] || !c->c_h[q] || !c->ik_h[q] || !c->b_e[q] || !c->c_e[q] || !c->ik_e[q])
            return fail(FDTD_ERR_INVALID, "CPML profile pointer for axis %d is NULL", q);
    if (gb) {
        if ((rc = check_span(g, gb->lo, gb->hi, "gradient box"))) return rc;
        if (!gb->e_next || !gb->e_prev || !gb->g)
            return fail(FDTD_ERR_INVALID, "gradient box buffer is NULL");
    }
    fdtd::AdjSeed sd;
    if ((rc = build_seed(g, next_seed, sd))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    int nnext = 0;
    for (int q = 0; q < 3; ++q) nnext += (a->E_next[q] != nullptr) + (a->H_next[q] != nullptr);
    if (nnext != 0 && nnext != 6)
        return fail(FDTD_ERR_INVALID, "E_next/H_next must be all set or all NULL");
    if (nnext == 6) {
        for (int q = 0; q < 3; ++q)
            for (int r = 0; r < 3; ++r)
                if (a->E_next[q] == a->E[r] || a->H_next[q] == a->H[r] ||
                    a->E_next[q] == a->H[r] || a->H_next[q] == a->E[r])
                    return fail(FDTD_ERR_INVALID, "E_next/H_next must not alias E/H");
        if (g->dtype == FDTD_F32)
            return cuda_status(fdtd::launch_adjoint_step_fused<float>(
                                   make_adj<float>(g, a, c), make_grad<float>(gb), sd,
                                   adj_out<float>(a), st),
                               "adjoint_step");
        return cuda_status(fdtd::launch_adjoint_step_fused<double>(
                               make_adj<double>(g, a, c), make_grad<double>(gb), sd,
                               adj_out<double>(a), st),
                           "adjoint_step");
    }
    if (g->dtype == FDTD_F32)
        return cuda_status(fdtd::launch_adjoint_step<float>(make_adj<float>(g, a, c),
                                                            make_grad<float>(gb), sd, st),
                           "adjoint_step");
    return cuda_status(fdtd::launch_adjoint_step<double>(make_adj<double>(g, a, c),
                                                         make_grad<double>(gb), sd, st),
                       "adjoint_step");
}

int fdtd_profile_steps(int32_t enable) {
    fdtd::profile_enable(enable != 0);
    return FDTD_OK;
}

int fdtd_profile_read(double ms[5], int32_t *nsteps) {
    if (!ms || !nsteps) return fail(FDTD_ERR_INVALID, "NULL output");
    int n = 0;
    cudaError_t e = fdtd::profile_read(ms, &n);
    *nsteps = n;
    return cuda_status(e, "profile_read");
}

int64_t fdtd_launch_count(void) { return fdtd::g_launches.load(std::memory_order_relaxed); }

int fdtd_set_epsilon(const fdtd_grid *g, const void *eps, const void *sigma, int32_t eps_dtype,
                     double dt, double eps0, void *const ce[3], void *const ca[3], void *stream) {
    int rc;
    if ((rc = check_grid(g))) return rc;
    if (!eps || !ce || !ce[0] || !ce[1] || !ce[2]) return fail(FDTD_ERR_INVALID, "NULL buffer");
    if (sigma && (!ca || !ca[0] || !ca[1] || !ca[2]))
        return fail(FDTD_ERR_INVALID, "sigma given without ca outputs");
    if (eps_dtype != FDTD_F32 && eps_dtype != FDTD_F64)
        return fail(FDTD_ERR_INVALID, "eps_dtype must be FDTD_F32 or FDTD_F64, got %d", eps_dtype);
    if (!(dt > 0) || !(eps0 > 0)) return fail(FDTD_ERR_INVALID, "dt and eps0 must be positive");
    fdtd::MatScalars m;
    m.scale = dt / eps0;
    m.dt = dt;
    m.two_eps0 = 2.0 * eps0;
    m.eps0 = eps0;
    cudaStream_t st = (cudaStream_t)stream;
    void *const nul[3] = {nullptr, nullptr, nullptr};
    void *const *cav = sigma ? ca : nul;
    cudaError_t e;
    if (g->dtype == FDTD_F32) {
        if (eps_dtype == FDTD_F32)
            e = fdtd::launch_edge_coeffs<float, float>(g->nx, g->ny, g->nz, (const float *)eps,
                                                       (const float *)sigma, m, (float *const *)ce,
                                                       (float *const *)cav, st);
        else
            e = fdtd::launch_edge_coeffs<float, double>(g->nx, g->ny, g->nz, (const double *)eps,
                                                        (const double *)sigma, m,
                                                        (float *const *)ce, (float *const *)cav, st);
    } else {
        if (eps_dtype == FDTD_F32)
            e = fdtd::launch_edge_coeffs<double, float>(g->nx, g->ny, g->nz, (const float *)eps,
                                                        (const float *)sigma, m,
                                                        (double *const *)ce, (double *const *)cav,
                                                        st);
        else
            e = fdtd::launch_edge_coeffs<double, double>(g->nx, g->ny, g->nz,
                                                         (const double *)eps,
                                                         (const double *)sigma, m,
                                                         (double *const *)ce,
                                                         (double *const *)cav, st);
    }
    return cuda_status(e, "set_epsilon");
}

int fdtd_n2f_workspace(const fdtd_n2f_face *faces, int32_t nfaces, int32_t nfreq, int32_t n_obs,
                       int32_t mode, uint64_t *bytes) {
    if (!bytes) return fail(FDTD_ERR_INVALID, "bytes is NULL");
    N2FPlan pl;
    int rc;
    if ((rc = plan_n2f(faces, nfaces, nfreq, n_obs, mode, pl))) return rc;
    *bytes = pl.total;
    return FDTD_OK;
}

int fdtd_n2f_contract(const fdtd_n2f_face *faces, int32_t nfaces, int32_t cur_dtype,
                      const double *freqs, int32_t nfreq, const double *dirs, int32_t n_obs,
                      int32_t mode, void *workspace, uint64_t workspace_bytes, void *nl,
                      void *stream) {
    N2FPlan pl;
    int rc;
    if ((rc = plan_n2f(faces, nfaces, nfreq, n_obs, mode, pl))) return rc;
    if (cur_dtype != FDTD_F32 && cur_dtype != FDTD_F64)
        return fail(FDTD_ERR_INVALID, "cur_dtype must be FDTD_F32 or FDTD_F64, got %d", cur_dtype);
    if (!freqs || !dirs || !nl) return fail(FDTD_ERR_INVALID, "NULL buffer");
    auto &P = pl.P;
    P.dirs = dirs;
    P.freqs = freqs;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    if (mode == FDTD_N2F_FP64) {
        e = cur_dtype == FDTD_F32 ? fdtd::n2f::launch_fp64<float2>(P, nfreq, (double2 *)nl, st)
                                  : fdtd::n2f::launch_fp64<double2>(P, nfreq, (double2 *)nl, st);
        return cuda_status(e, "n2f_contract");
    }
    if (!workspace || workspace_bytes < pl.total)
        return fail(FDTD_ERR_INVALID, "workspace of %llu bytes is smaller than the %llu needed",
                    (unsigned long long)workspace_bytes, (unsigned long long)pl.total);
    if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
        return fail(FDTD_ERR_INVALID, "workspace must be 256-byte aligned");
    unsigned char *ws = (unsigned char *)workspace;
    for (int f = 0; f < nfaces; ++f) {
        const auto &G = P.face[f];
        e = cur_dtype == FDTD_F32
                ? fdtd::n2f::launch_pack<float2>(mode, (const float2 *)P.cur[f], nfreq, G.np, G.nq,
                                                 G.ks, G.nt, ws + G.b_off, st)
                : fdtd::n2f::launch_pack<double2>(mode, (const double2 *)P.cur[f], nfreq, G.np,
                                                  G.nq, G.ks, G.nt, ws + G.b_off, st);
        if (e != cudaSuccess) return cuda_status(e, "n2f_pack");
    }
    P.btiles = ws;
    P.partial = (float2 *)(ws + pl.partial_off);
    if ((e = fdtd::n2f::launch_contract(mode, P, nfreq, st)) != cudaSuccess)
        return cuda_status(e, "n2f_contract");
    return cuda_status(fdtd::n2f::launch_combine(P, nfreq, (float2 *)nl, st), "n2f_combine");
}

int fdtd_farfield_eh(const void *nl, int32_t nl_dtype, const double *obs_xyz, int32_t n_obs,
                     double k_wave, double eta0, double *eh, void *stream) {
    if (!nl || !obs_xyz || !eh) return fail(FDTD_ERR_INVALID, "NULL buffer");
    if (n_obs <= 0) return fail(FDTD_ERR_INVALID, "n_obs must be positive, got %d", n_obs);
    if (nl_dtype != FDTD_F32 && nl_dtype != FDTD_F64)
        return fail(FDTD_ERR_INVALID, "nl_dtype must be FDTD_F32 or FDTD_F64, got %d", nl_dtype);
    if (!(k_wave >= 0) || !(eta0 > 0)) return fail(FDTD_ERR_INVALID, "k_wave, eta0 must be positive");
    return cuda_status(fdtd::launch_farfield_eh(nl, nl_dtype == FDTD_F64, obs_xyz, n_obs, k_wave,
                                                eta0, eh, (cudaStream_t)stream),
                       "farfield_eh");
}

}  // extern "C"
