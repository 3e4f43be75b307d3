// TMA / mbarrier helpers shared by the plane-marching kernels (the forward
// interior kernel in yee_fused.cu and the adjoint interior kernel in
// adjoint_fused.cu), the host-side tensor-map cache and the per-thread side
// stream on which CPML-shell kernels run beside them.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

namespace fdtd {

template <typename T>
struct VecT;
template <>
struct VecT<float> {
    using type = float4;
};
template <>
struct VecT<double> {
    using type = double2;
};

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

__device__ __forceinline__ bool mbar_test_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int c0, int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

template <typename T, int V>
__device__ __forceinline__ void ld_vec(const T *p, T (&out)[V]) {
    using VT = typename VecT<T>::type;
    const VT v = *reinterpret_cast<const VT *>(p);
    const T *q = reinterpret_cast<const T *>(&v);
#pragma unroll
    for (int e = 0; e < V; ++e) out[e] = q[e];
}

template <typename T, int V>
__device__ __forceinline__ void st_vec(T *p, const T (&in)[V]) {
    using VT = typename VecT<T>::type;
    VT v;
    T *q = reinterpret_cast<T *>(&v);
#pragma unroll
    for (int e = 0; e < V; ++e) q[e] = in[e];
    *reinterpret_cast<VT *>(p) = v;
}


// 3-D tiled tensor map (x = z-index fastest, y = j, z = i) of an (nx, ny, nz)
// array of elem-byte values with a box of b0 x b1 x 1, no swizzle, no
// multicast; cached by (base, shape, elem, box, promotion).  l2_promote: the L2
// fetch granularity of the copies in bytes (256, 128, 64; 0 = none, for boxes
// whose rows are short runs that neighbouring tiles do not share).  False if
// the driver's encoder is unavailable or rejects the map.
bool make_tensor_map(CUtensorMap *out, const void *base, int nx, int ny, int nz, int elem,
                     int b0, int b1, int l2_promote = 256);

// Host-side caches that keep the per-step launch path short (an engine calls
// the step with the same buffers, alternating between two parities):
//   KeyedCache : the last few values built for a key of NW 64-bit words (the
//                tensor maps of one buffer set), one lock per lookup;
//   device_sm_count : the SM count of the current device, queried once;
//   ensure_max_dynamic_smem : cudaFuncSetAttribute(MaxDynamicSharedMemorySize)
//                only when the kernel's current limit is below the size.
template <typename V, int NW, int NE = 4>
class KeyedCache {
  public:
    bool get(const uint64_t (&key)[NW], V &out) {
        std::lock_guard<std::mutex> lk(mu_);
        for (int q = 0; q < n_; ++q)
            if (memcmp(keys_[q], key, sizeof(key)) == 0) {
                out = vals_[q];
                return true;
            }
        return false;
    }
    void put(const uint64_t (&key)[NW], const V &v) {
        std::lock_guard<std::mutex> lk(mu_);
        const int q = n_ < NE ? n_++ : (int)(next_++ % NE);
        memcpy(keys_[q], key, sizeof(key));
        vals_[q] = v;
    }

  private:
    std::mutex mu_;
    uint64_t keys_[NE][NW];
    V vals_[NE];
    int n_ = 0;
    unsigned next_ = 0;
};

int device_sm_count();
cudaError_t ensure_max_dynamic_smem(const void *func, int bytes);

// A stream of this host thread and device, with events to fork from and join
// back to a caller's stream.  slot 0 serves the forward step, slot 1 the
// adjoint step, so the two can run on different caller streams concurrently.
struct SideStream {
    cudaStream_t s = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
cudaError_t side_stream(SideStream **out, int slot = 0);

}  // namespace fdtd
