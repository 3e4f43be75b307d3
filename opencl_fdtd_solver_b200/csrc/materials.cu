// Yee-edge material coefficients on the device (set_epsilon without a host pass).
//
// Restates, per edge, the reference host math of opencl_fdtd_solver/materials.py:
//   ε_edge = 0.5·(ε_i + ε_{i+1}) along the stagger axis, the last plane keeping
//   the cell value (:28-41);  ce = (dt/ε0)/ε_edge rounded once (:45-55);
//   lossy: loss = (σ_e·dt)/((2ε0)·ε_e), ca = (1 − loss)/(1 + loss),
//   cb = (dt/(ε0·ε_e))/(1 + loss) (:59-88).
// Every operation is a float64 IEEE operation in that order (the file is built
// with --fmad=false), so the rounded coefficients equal the host's bit for bit.
#include <cuda_runtime.h>

#include <cstdint>

#include "launch_count.cuh"

namespace fdtd {

// dt/eps0, dt, 2*eps0, eps0 (computed once on the host)
struct MatScalars {
    double scale, dt, two_eps0, eps0;
};

template <typename S>
__device__ __forceinline__ double edge_mean(const S *a, int64_t idx, int64_t stride, bool last) {
    const double v = (double)a[idx];
    if (last) return v;
    return 0.5 * (v + (double)a[idx + stride]);
}

template <typename T, typename S>
__global__ void k_edge_coeffs(int nx, int ny, int nz, const S *eps, const S *sigma,
                              MatScalars m, T *ce0, T *ce1, T *ce2, T *ca0, T *ca1, T *ca2) {
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t sx = (int64_t)ny * nz, sy = nz;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(q % nz);
        const int64_t t = q / nz;
        const int j = (int)(t % ny);
        const int i = (int)(t / ny);
        const bool last[3] = {i == nx - 1, j == ny - 1, k == nz - 1};
        const int64_t st[3] = {sx, sy, 1};
        T *ce[3] = {ce0, ce1, ce2};
        T *ca[3] = {ca0, ca1, ca2};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double e = edge_mean(eps, q, st[c], last[c]);
            if (sigma == nullptr) {
                ce[c][q] = (T)(m.scale / e);
            } else {
                const double s = edge_mean(sigma, q, st[c], last[c]);
                const double loss = (s * m.dt) / (m.two_eps0 * e);
                const double denom = 1.0 + loss;
                ca[c][q] = (T)((1.0 - loss) / denom);
                ce[c][q] = (T)((m.dt / (m.eps0 * e)) / denom);
            }
        }
    }
}

template <typename T, typename S>
cudaError_t launch_edge_coeffs(int nx, int ny, int nz, const S *eps, const S *sigma,
                               const MatScalars &m, T *const ce[3], T *const ca[3],
                               cudaStream_t st) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t n = (int64_t)nx * ny * nz;
    const int thr = 256;
    int64_t blocks = (n + thr - 1) / thr;
    if (blocks > (int64_t)sms * 16) blocks = (int64_t)sms * 16;
    k_edge_coeffs<T, S><<<(unsigned)blocks, thr, 0, st>>>(nx, ny, nz, eps, sigma, m, ce[0], ce[1],
                                                          ce[2], ca[0], ca[1], ca[2]);
    count_launches(1);
    return cudaGetLastError();
}

template cudaError_t launch_edge_coeffs<float, float>(int, int, int, const float *, const float *,
                                                      const MatScalars &, float *const[3],
                                                      float *const[3], cudaStream_t);
template cudaError_t launch_edge_coeffs<float, double>(int, int, int, const double *,
                                                       const double *, const MatScalars &,
                                                       float *const[3], float *const[3],
                                                       cudaStream_t);
template cudaError_t launch_edge_coeffs<double, float>(int, int, int, const float *,
                                                       const float *, const MatScalars &,
                                                       double *const[3], double *const[3],
                                                       cudaStream_t);
template cudaError_t launch_edge_coeffs<double, double>(int, int, int, const double *,
                                                        const double *, const MatScalars &,
                                                        double *const[3], double *const[3],
                                                        cudaStream_t);

}  // namespace fdtd
