// Packed gather of field sub-boxes for host reads (fdtd_read_regions).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/fdtd_b200.h"

namespace fdtd {

struct RegionList {
    int n;
    int32_t lo[FDTD_MAX_REGIONS][3];
    int32_t ext[FDTD_MAX_REGIONS][3];   // hi - lo per axis
    int64_t off[FDTD_MAX_REGIONS + 1];  // packed offsets; off[n] = total cells
};

// Gather the boxes of `src` (C order, ny * nz per i plane) into `staging`, then
// copy the packed cells to `host` on `st`.
template <typename T>
cudaError_t launch_read_regions(const T *src, int ny, int nz, const RegionList &r, T *staging,
                                void *host, cudaStream_t st);

}  // namespace fdtd
