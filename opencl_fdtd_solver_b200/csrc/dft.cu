// Huygens-box face DFT, its relative-change reduction, and the float64
// far-field surface integral.
//
//   k_dft_faces      : dft_farfield.cl:116-230 (co-located tangential E/H,
//                      E at the step time, H half a step earlier), for nfreq
//                      frequencies per launch with complex128 accumulators.
//   k_rel_partial/.. : dft_farfield.cl:237-290 + the host sum of
//                      monitors.py:560-569, as a deterministic two-pass reduce.
//   k_farfield_nl    : dft_farfield.cl:372-556 (trapezoid weights, face-centre
//                      sample positions, N = n x H, L = -n x E), one block per
//                      observation point, block tree reduction (no atomics).
//   k_farfield_eh    : dft_farfield.cl:559-635 with the kernel's sign,
//                      E = -jk e^{-jkr}/(4 pi r) (eta N_t - r x L), H = -r x E / eta.
//
// Compiled with --fmad=false: the face averages and the accumulation round as
// the oracle does.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "launch_count.cuh"
#include "../../include/fdtd_b200.h"

namespace fdtd {

struct FaceCoord {
    int face, i, j, k;
};

__device__ __forceinline__ FaceCoord face_coord(const fdtd_box &b, int s) {
    const int nyf = b.iy1 - b.iy0 + 1, nzf = b.iz1 - b.iz0 + 1;
    FaceCoord c;
    if (s < b.off[1]) {
        const int loc = s - b.off[0];
        c = {0, b.ix0, b.iy0 + loc / nzf, b.iz0 + loc % nzf};
    } else if (s < b.off[2]) {
        const int loc = s - b.off[1];
        c = {1, b.ix1, b.iy0 + loc / nzf, b.iz0 + loc % nzf};
    } else if (s < b.off[3]) {
        const int loc = s - b.off[2];
        c = {2, b.ix0 + loc / nzf, b.iy0, b.iz0 + loc % nzf};
    } else if (s < b.off[4]) {
        const int loc = s - b.off[3];
        c = {3, b.ix0 + loc / nzf, b.iy1, b.iz0 + loc % nzf};
    } else if (s < b.off[5]) {
        const int loc = s - b.off[4];
        c = {4, b.ix0 + loc / nyf, b.iy0 + loc % nyf, b.iz0};
    } else {
        const int loc = s - b.off[5];
        c = {5, b.ix0 + loc / nyf, b.iy0 + loc % nyf, b.iz1};
    }
    return c;
}

template <typename T>
__global__ void k_dft_faces(int nx, int ny, int nz, const T *Ex, const T *Ey, const T *Ez,
                            const T *Hx, const T *Hy, const T *Hz, fdtd_box b, double *acc,
                            const double *phase) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.n_face) return;
    const FaceCoord c = face_coord(b, s);
    const int i = c.i, j = c.j, k = c.k;
    // the face's four tangential components (Ex..Hz numbering): x faces Ey, Ez,
    // Hy, Hz; y faces Ex, Ez, Hx, Hz; z faces Ex, Ey, Hx, Hy
    const int g = c.face >> 1;
    const int c0 = g == 0 ? 1 : 0, c1 = g == 2 ? 1 : 2, c2 = g == 0 ? 4 : 3, c3 = g == 2 ? 4 : 5;
    // one frequency per thread (blockIdx.y); the four accumulator loads are
    // issued first, before the field gathers, so they overlap one another and
    // the gathers instead of each waiting behind the previous store
    const int f = blockIdx.y;
    double2 *A = reinterpret_cast<double2 *>(acc);
    double2 *a0 = A + ((int64_t)c0 * b.nfreq + f) * b.n_face + s;
    double2 *a1 = A + ((int64_t)c1 * b.nfreq + f) * b.n_face + s;
    double2 *a2 = A + ((int64_t)c2 * b.nfreq + f) * b.n_face + s;
    double2 *a3 = A + ((int64_t)c3 * b.nfreq + f) * b.n_face + s;
    double2 q0 = *a0, q1 = *a1, q2 = *a2, q3 = *a3;
    auto at = [&](const T *F, int ii, int jj, int kk) {
        return F[((int64_t)ii * ny + jj) * nz + kk];
    };
    const T half = T(0.5), quarter = T(0.25);
    T t0, t1, t2, t3;  // the tangential values in the order c0..c3
    if (c.face <= 1) {
        const int k1 = (k + 1 < nz) ? k + 1 : k, j1 = (j + 1 < ny) ? j + 1 : j;
        const int ilo = (i > 0) ? i - 1 : i;
        t0 = (k1 != k) ? half * (at(Ey, i, j, k) + at(Ey, i, j, k1)) : at(Ey, i, j, k);
        t1 = (j1 != j) ? half * (at(Ez, i, j, k) + at(Ez, i, j1, k)) : at(Ez, i, j, k);
        t2 = quarter * (at(Hy, i, j, k) + at(Hy, ilo, j, k) + at(Hy, i, j1, k) + at(Hy, ilo, j1, k));
        t3 = quarter * (at(Hz, i, j, k) + at(Hz, ilo, j, k) + at(Hz, i, j, k1) + at(Hz, ilo, j, k1));
    } else if (c.face <= 3) {
        const int i1 = (i + 1 < nx) ? i + 1 : i, k1 = (k + 1 < nz) ? k + 1 : k;
        const int jlo = (j > 0) ? j - 1 : j;
        t0 = (k1 != k) ? half * (at(Ex, i, j, k) + at(Ex, i, j, k1)) : at(Ex, i, j, k);
        t1 = (i1 != i) ? half * (at(Ez, i, j, k) + at(Ez, i1, j, k)) : at(Ez, i, j, k);
        t2 = quarter * (at(Hx, i, j, k) + at(Hx, i, jlo, k) + at(Hx, i1, j, k) + at(Hx, i1, jlo, k));
        t3 = quarter * (at(Hz, i, j, k) + at(Hz, i, jlo, k) + at(Hz, i, j, k1) + at(Hz, i, jlo, k1));
    } else {
        const int i1 = (i + 1 < nx) ? i + 1 : i, j1 = (j + 1 < ny) ? j + 1 : j;
        const int klo = (k > 0) ? k - 1 : k;
        t0 = (j1 != j) ? half * (at(Ex, i, j, k) + at(Ex, i, j1, k)) : at(Ex, i, j, k);
        t1 = (i1 != i) ? half * (at(Ey, i, j, k) + at(Ey, i1, j, k)) : at(Ey, i, j, k);
        t2 = quarter * (at(Hx, i, j, k) + at(Hx, i, j, klo) + at(Hx, i, j1, k) + at(Hx, i, j1, klo));
        t3 = quarter * (at(Hy, i, j, k) + at(Hy, i, j, klo) + at(Hy, i1, j, k) + at(Hy, i1, j, klo));
    }
    // E samples take the E phase of the step, H samples the H phase
    const double epr = phase[4 * f], epi = phase[4 * f + 1];
    const double hpr = phase[4 * f + 2], hpi = phase[4 * f + 3];
    const double v0 = (double)t0, v1 = (double)t1, v2 = (double)t2, v3 = (double)t3;
    q0.x = q0.x + v0 * epr;
    q0.y = q0.y + v0 * epi;
    q1.x = q1.x + v1 * epr;
    q1.y = q1.y + v1 * epi;
    q2.x = q2.x + v2 * hpr;
    q2.y = q2.y + v2 * hpi;
    q3.x = q3.x + v3 * hpr;
    q3.y = q3.y + v3 * hpi;
    *a0 = q0;
    *a1 = q1;
    *a2 = q2;
    *a3 = q3;
}

constexpr int REL_THREADS = 256;

__global__ void k_rel_partial(const double2 *cur, const double2 *prev, int n, int nfreq, int fi,
                              double *scratch) {
    __shared__ double sn[REL_THREADS], sd[REL_THREADS];
    double num = 0.0, den = 0.0;
    for (int s = blockIdx.x * REL_THREADS + threadIdx.x; s < n; s += gridDim.x * REL_THREADS) {
        for (int comp = 0; comp < 6; ++comp) {
            const int64_t o = ((int64_t)comp * nfreq + fi) * n + s;
            const double2 c = cur[o], p = prev[o];
            const double dx = c.x - p.x, dy = c.y - p.y;
            num += dx * dx + dy * dy;
            den += c.x * c.x + c.y * c.y;
        }
    }
    sn[threadIdx.x] = num;
    sd[threadIdx.x] = den;
    __syncthreads();
    for (int st = REL_THREADS / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) {
            sn[threadIdx.x] += sn[threadIdx.x + st];
            sd[threadIdx.x] += sd[threadIdx.x + st];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        scratch[2 * blockIdx.x] = sn[0];
        scratch[2 * blockIdx.x + 1] = sd[0];
    }
}

__global__ void k_rel_final(const double *scratch, int nblk, double *out2) {
    __shared__ double sn[REL_THREADS], sd[REL_THREADS];
    double num = 0.0, den = 0.0;
    for (int b = threadIdx.x; b < nblk; b += REL_THREADS) {
        num += scratch[2 * b];
        den += scratch[2 * b + 1];
    }
    sn[threadIdx.x] = num;
    sd[threadIdx.x] = den;
    __syncthreads();
    for (int st = REL_THREADS / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) {
            sn[threadIdx.x] += sn[threadIdx.x + st];
            sd[threadIdx.x] += sd[threadIdx.x + st];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out2[0] = sn[0];
        out2[1] = sd[0];
    }
}

constexpr int FF_THREADS = 256;

// One block per observation point: NL[obs][6] (N xyz, L xyz), complex128.
__global__ void __launch_bounds__(FF_THREADS)
    k_farfield_nl(fdtd_box b, const double2 *acc, int fi, double dl, double k_wave,
                  const double *obs, int n_obs, double2 *nl) {
    const int o = blockIdx.x;
    if (o >= n_obs) return;
    const double ox = obs[3 * o], oy = obs[3 * o + 1], oz = obs[3 * o + 2];
    double r = sqrt(ox * ox + oy * oy + oz * oz);
    if (r < 1e-30) r = 1e-30;
    const double rx = ox / r, ry = oy / r, rz = oz / r;
    const double dA = dl * dl;
    double accr[6] = {0, 0, 0, 0, 0, 0}, acci[6] = {0, 0, 0, 0, 0, 0};
    const int64_t stride = (int64_t)b.nfreq * b.n_face;
    for (int s = threadIdx.x; s < b.n_face; s += FF_THREADS) {
        const FaceCoord c = face_coord(b, s);
        double xp, yp, zp, wj, wk;
        if (c.face <= 1) {
            xp = c.i * dl;
            yp = (c.j + 0.5) * dl;
            zp = (c.k + 0.5) * dl;
            wj = (c.j == b.iy0 || c.j == b.iy1) ? 0.5 : 1.0;
            wk = (c.k == b.iz0 || c.k == b.iz1) ? 0.5 : 1.0;
        } else if (c.face <= 3) {
            xp = (c.i + 0.5) * dl;
            yp = c.j * dl;
            zp = (c.k + 0.5) * dl;
            wj = (c.i == b.ix0 || c.i == b.ix1) ? 0.5 : 1.0;
            wk = (c.k == b.iz0 || c.k == b.iz1) ? 0.5 : 1.0;
        } else {
            xp = (c.i + 0.5) * dl;
            yp = (c.j + 0.5) * dl;
            zp = c.k * dl;
            wj = (c.i == b.ix0 || c.i == b.ix1) ? 0.5 : 1.0;
            wk = (c.j == b.iy0 || c.j == b.iy1) ? 0.5 : 1.0;
        }
        const double ph = k_wave * (rx * xp + ry * yp + rz * zp);
        double sn, cs;
        sincos(ph, &sn, &cs);
        const double w = dA * wj * wk;
        const double nf = (c.face & 1) ? 1.0 : -1.0;
        auto g = [&](int comp) { return acc[comp * stride + (int64_t)fi * b.n_face + s]; };
        // contribution cur * e^{j ph} * w into output component oc
        auto add = [&](int oc, double sign, double2 v) {
            const double re = sign * v.x, im = sign * v.y;
            accr[oc] += (re * cs - im * sn) * w;
            acci[oc] += (re * sn + im * cs) * w;
        };
        if (c.face <= 1) {
            add(1, nf, g(5));    // Ny +=  n Hz
            add(2, -nf, g(4));   // Nz += -n Hy
            add(4, -nf, g(2));   // Ly += -n Ez
            add(5, nf, g(1));    // Lz +=  n Ey
        } else if (c.face <= 3) {
            add(0, -nf, g(5));   // Nx += -n Hz
            add(2, nf, g(3));    // Nz +=  n Hx
            add(3, nf, g(2));    // Lx +=  n Ez
            add(5, -nf, g(0));   // Lz += -n Ex
        } else {
            add(0, nf, g(4));    // Nx +=  n Hy
            add(1, -nf, g(3));   // Ny += -n Hx
            add(3, -nf, g(1));   // Lx += -n Ey
            add(4, nf, g(0));    // Ly +=  n Ex
        }
    }
    __shared__ double red[2 * 6][FF_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int q = 0; q < 6; ++q) {
        double a = accr[q], bq = acci[q];
        for (int off = 16; off > 0; off >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, off);
            bq += __shfl_down_sync(0xffffffffu, bq, off);
        }
        if (lane == 0) {
            red[2 * q][wid] = a;
            red[2 * q + 1][wid] = bq;
        }
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        double s = 0.0;
        for (int w = 0; w < FF_THREADS / 32; ++w) s += red[threadIdx.x][w];
        double *out = reinterpret_cast<double *>(nl + 6 * (int64_t)o);
        out[threadIdx.x] = s;
    }
}

// NL may be complex128 (the direct sums) or complex64 (the tensor-core contraction).
template <typename NT>
__global__ void k_farfield_eh(const NT *nl, const double *obs, int n_obs, double k_wave,
                              double eta0, double2 *eh) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_obs) return;
    const double ox = obs[3 * p], oy = obs[3 * p + 1], oz = obs[3 * p + 2];
    double r = sqrt(ox * ox + oy * oy + oz * oz);
    if (r < 1e-30) r = 1e-30;
    const double rh[3] = {ox / r, oy / r, oz / r};
    double2 N[3], L[3];
    for (int c = 0; c < 3; ++c) {
        const NT n = nl[6 * (int64_t)p + c], l = nl[6 * (int64_t)p + 3 + c];
        N[c] = make_double2((double)n.x, (double)n.y);
        L[c] = make_double2((double)l.x, (double)l.y);
    }
    double sn, cs;
    sincos(k_wave * r, &sn, &cs);
    const double scale = k_wave / (4.0 * 3.14159265358979323846 * r);
    // pref = (-j scale) * e^{-jkr} = (-j scale)(cs - j sn) = -scale sn - j scale cs
    const double pr = -scale * sn, pi = -scale * cs;
    const double ndr = rh[0] * N[0].x + rh[1] * N[1].x + rh[2] * N[2].x;
    const double ndi = rh[0] * N[0].y + rh[1] * N[1].y + rh[2] * N[2].y;
    double2 rxL[3];
    rxL[0] = make_double2(rh[1] * L[2].x - rh[2] * L[1].x, rh[1] * L[2].y - rh[2] * L[1].y);
    rxL[1] = make_double2(rh[2] * L[0].x - rh[0] * L[2].x, rh[2] * L[0].y - rh[0] * L[2].y);
    rxL[2] = make_double2(rh[0] * L[1].x - rh[1] * L[0].x, rh[0] * L[1].y - rh[1] * L[0].y);
    double2 E[3];
    for (int c = 0; c < 3; ++c) {
        const double ntr = N[c].x - ndr * rh[c], nti = N[c].y - ndi * rh[c];
        const double tr = eta0 * ntr - rxL[c].x, ti = eta0 * nti - rxL[c].y;
        E[c] = make_double2(pr * tr - pi * ti, pr * ti + pi * tr);
    }
    double2 *out = eh + 6 * (int64_t)p;
    out[0] = E[0];
    out[1] = E[1];
    out[2] = E[2];
    out[3] = make_double2(-(rh[1] * E[2].x - rh[2] * E[1].x) / eta0,
                          -(rh[1] * E[2].y - rh[2] * E[1].y) / eta0);
    out[4] = make_double2(-(rh[2] * E[0].x - rh[0] * E[2].x) / eta0,
                          -(rh[2] * E[0].y - rh[0] * E[2].y) / eta0);
    out[5] = make_double2(-(rh[0] * E[1].x - rh[1] * E[0].x) / eta0,
                          -(rh[0] * E[1].y - rh[1] * E[0].y) / eta0);
}

template <typename T>
cudaError_t launch_dft_faces(int nx, int ny, int nz, const T *const E[3], const T *const H[3],
                             const fdtd_box &b, double *acc, const double *phase,
                             cudaStream_t st) {
    const int thr = 128;
    const dim3 grid((unsigned)((b.n_face + thr - 1) / thr), (unsigned)b.nfreq, 1);
    k_dft_faces<T><<<grid, thr, 0, st>>>(nx, ny, nz, E[0], E[1], E[2], H[0], H[1], H[2], b, acc,
                                         phase);
    count_launches(1);
    return cudaGetLastError();
}
template cudaError_t launch_dft_faces<float>(int, int, int, const float *const[3],
                                             const float *const[3], const fdtd_box &,
                                             double *, const double *, cudaStream_t);
template cudaError_t launch_dft_faces<double>(int, int, int, const double *const[3],
                                              const double *const[3], const fdtd_box &,
                                              double *, const double *, cudaStream_t);

int rel_change_blocks(int n) {
    int b = (n + REL_THREADS - 1) / REL_THREADS;
    return b < 1 ? 1 : (b > 1024 ? 1024 : b);
}

cudaError_t launch_rel_change(const double *cur, const double *prev, int n, int nfreq, int fi,
                              double *scratch, double *out2, cudaStream_t st) {
    const int nb = rel_change_blocks(n);
    k_rel_partial<<<nb, REL_THREADS, 0, st>>>(reinterpret_cast<const double2 *>(cur),
                                              reinterpret_cast<const double2 *>(prev), n, nfreq,
                                              fi, scratch);
    count_launches(1);
    k_rel_final<<<1, REL_THREADS, 0, st>>>(scratch, nb, out2);
    count_launches(1);
    return cudaGetLastError();
}

// ---- relative change without caller-provided scratch ---------------------
//
// Same two-pass reduction as launch_rel_change, but the per-block partial sums
// live in this file-scope device array instead of a buffer the caller
// allocates.  It holds NOALLOC_REL_BLOCKS blocks (16 KiB of doubles) on every
// GPU that loads the library, for the life of the process.  One partial per
// block of 256 face samples, so n_face is limited to NOALLOC_REL_BLOCKS * 256.
// Each call writes every partial it reads back, so nothing needs clearing
// between calls; calls that overlap on the GPU share the array and race.
constexpr int NOALLOC_REL_BLOCKS = 1024;
static_assert(NOALLOC_REL_BLOCKS * REL_THREADS == FDTD_NOALLOC_MAX_FACE,
              "the built-in scratch array must hold FDTD_NOALLOC_MAX_FACE face samples");
static __device__ __align__(256) double g_rel_scratch[2 * NOALLOC_REL_BLOCKS];

int noalloc_rel_max_face() { return NOALLOC_REL_BLOCKS * REL_THREADS; }

namespace {
std::mutex g_scratch_mu;
double *g_scratch_ptr[256];  // last resolved device address of g_rel_scratch, per device
}  // namespace

// Device address of the scratch array on the current device.  Host code must
// not use the array's name as a device pointer (it is only a host-side
// stand-in), so the address comes from cudaGetSymbolAddress, with that device
// current.  It is looked up again on every call made while `st` is not being
// captured, so a device reset (which reloads the module and may move the array)
// cannot leave a stale address behind; during a capture the address from the
// device's last uncaptured call is used, and a capture before any such call is
// refused.
cudaError_t noalloc_rel_scratch(cudaStream_t st, double **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if ((e = cudaStreamIsCapturing(st, &cs)) != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (cs == cudaStreamCaptureStatusNone) {
        void *p = nullptr;
        if ((e = cudaGetSymbolAddress(&p, g_rel_scratch)) != cudaSuccess) return e;
        g_scratch_ptr[dev] = static_cast<double *>(p);
    } else if (!g_scratch_ptr[dev]) {
        return cudaErrorStreamCaptureUnsupported;
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

cudaError_t launch_rel_change_noalloc(const double *cur, const double *prev, int n, int nfreq,
                                      int fi, double *out2, cudaStream_t st) {
    double *scratch = nullptr;
    cudaError_t e = noalloc_rel_scratch(st, &scratch);
    if (e != cudaSuccess) return e;
    const int nb = (n + REL_THREADS - 1) / REL_THREADS;
    k_rel_partial<<<nb, REL_THREADS, 0, st>>>(reinterpret_cast<const double2 *>(cur),
                                              reinterpret_cast<const double2 *>(prev), n, nfreq,
                                              fi, scratch);
    count_launches(1);
    k_rel_final<<<1, REL_THREADS, 0, st>>>(scratch, nb, out2);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_farfield(const fdtd_box &b, const double *acc, int fi, double dl,
                            double k_wave, double eta0, const double *obs, int n_obs,
                            double *nl, double *eh, cudaStream_t st) {
    k_farfield_nl<<<n_obs, FF_THREADS, 0, st>>>(b, reinterpret_cast<const double2 *>(acc), fi,
                                                dl, k_wave, obs, n_obs,
                                                reinterpret_cast<double2 *>(nl));
    count_launches(1);
    k_farfield_eh<double2><<<(n_obs + 127) / 128, 128, 0, st>>>(reinterpret_cast<const double2 *>(nl),
                                                       obs, n_obs, k_wave, eta0,
                                                       reinterpret_cast<double2 *>(eh));
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_farfield_eh(const void *nl, int nl_f64, const double *obs, int n_obs,
                               double k_wave, double eta0, double *eh, cudaStream_t st) {
    const unsigned nb = (unsigned)((n_obs + 127) / 128);
    if (nl_f64)
        k_farfield_eh<double2><<<nb, 128, 0, st>>>(reinterpret_cast<const double2 *>(nl), obs, n_obs,
                                                   k_wave, eta0, reinterpret_cast<double2 *>(eh));
    else
        k_farfield_eh<float2><<<nb, 128, 0, st>>>(reinterpret_cast<const float2 *>(nl), obs, n_obs,
                                                  k_wave, eta0, reinterpret_cast<double2 *>(eh));
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace fdtd
