// Gather of field sub-boxes into one packed device buffer, ahead of a single
// device-to-host copy (fdtd_read_regions).  A host monitor that reads a few
// planes of each field per step then moves those planes, not the volume.
#include <cuda_runtime.h>

#include <cstdint>

#include "hostio.cuh"
#include "launch_count.cuh"

namespace fdtd {

// blockIdx.y selects the box; the x blocks stride over its cells in C order, so
// consecutive threads read consecutive k and write consecutive packed slots.
template <typename T>
__global__ void __launch_bounds__(256) k_gather_regions(const T *__restrict__ src, int ny, int nz,
                                                        const __grid_constant__ RegionList r,
                                                        T *__restrict__ dst) {
    const int q = blockIdx.y;
    const int64_t cnt = r.off[q + 1] - r.off[q];
    const int ej = r.ext[q][1], ek = r.ext[q][2];
    const int64_t plane = (int64_t)ej * ek;
    T *out = dst + r.off[q];
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < cnt;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = t / plane;
        const int64_t rem = t - a * plane;
        const int64_t b = rem / ek;
        const int64_t c = rem - b * ek;
        const int64_t i = r.lo[q][0] + a, j = r.lo[q][1] + b, k = r.lo[q][2] + c;
        out[t] = src[(i * ny + j) * nz + k];
    }
}

template <typename T>
cudaError_t launch_read_regions(const T *src, int ny, int nz, const RegionList &r, T *staging,
                                void *host, cudaStream_t st) {
    int64_t biggest = 0;
    for (int q = 0; q < r.n; ++q) {
        const int64_t c = r.off[q + 1] - r.off[q];
        if (c > biggest) biggest = c;
    }
    const int64_t total = r.off[r.n];
    if (total == 0) return cudaSuccess;
    // 148 SMs x 8 resident blocks of 256 threads covers the largest box in one
    // or a few grid-stride passes; small boxes get only the blocks they need.
    const int64_t want = (biggest + 255) / 256;
    const unsigned gx = (unsigned)(want < 148 * 8 ? (want > 0 ? want : 1) : 148 * 8);
    k_gather_regions<T><<<dim3(gx, (unsigned)r.n), 256, 0, st>>>(src, ny, nz, r, staging);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    count_launches(1);
    return cudaMemcpyAsync(host, staging, (size_t)total * sizeof(T), cudaMemcpyDeviceToHost, st);
}

template cudaError_t launch_read_regions<float>(const float *, int, int, const RegionList &,
                                                float *, void *, cudaStream_t);
template cudaError_t launch_read_regions<double>(const double *, int, int, const RegionList &,
                                                 double *, void *, cudaStream_t);

}  // namespace fdtd
